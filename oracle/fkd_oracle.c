/*
 * fkd_oracle.c -- CPU restatement of the FKDTree build and box searches.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the
 * product library (fkdtree_b200/libfkdtree_b200.so).  Only tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py load it.
 *
 * What it restates (reference paths are relative to the te42kyfo/FKDTree tree):
 *   fkd_oracle_build          FKDTree_cpu.h:221-277  (level-by-level nth_element build)
 *     partition_complete      FKDTree_cpu.h:287-296
 *     key order               FKDTree_cpu.h:246-252  (coordinate, then id on ties)
 *     add_at_position         FKDTree_cpu.h:280-285
 *   search variant 0          FKDTree_cpu.h:123-169  (search_in_the_box, level order)
 *   search variant 1          FKDTree_cpu.h:72-121   (search_in_the_box_BFS)
 *   search variant 2          FKDTree_cpu.h:25-70    (search_in_the_box_branchless)
 *   search variant 3          FKDTree_cpu.h:171-207  (search_in_the_box_recursive)
 *   search variant 4          FKDTree.h:54-86        (test_correct_search brute force)
 *   intersects / is_in_the_box FKDTree_cpu.h:302-321
 *
 * Differences from the reference, all deliberate:
 *   - the level-order / BFS / branchless frontiers grow without bound instead of
 *     using FQueue's fixed 1024-slot ring (FQueue.h:158, :232), so they stay
 *     correct where the reference would assert; the largest frontier occupancy
 *     FQueue would have needed is reported so callers can tell when the
 *     reference itself can run a query;
 *   - std::nth_element (libstdc++ introselect) is replaced by a plain
 *     quickselect.  Because the comparator is a strict total order when ids are
 *     unique, the selected element and the membership of both sides do not
 *     depend on the selection algorithm, so the produced tables are the same.
 *
 * Parity of this file is pinned against the reference itself: oracle/Makefile
 * compiles oracle/ref_harness.cpp against the unmodified reference headers into
 * oracle/_ref/libfkdref.so, and tests/golden/make_golden.py records its outputs
 * as the fixtures under tests/golden/ that tests/test_oracle.py checks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FKDO_MAXDIM 8

static unsigned floor_log2_u32(uint32_t x) { return 31u - (unsigned)__builtin_clz(x | 1u); }

/* FKDTree_cpu.h:287-296 */
static uint32_t partition_complete(uint32_t length) {
  if (length == 1) return 0;
  uint32_t index = 1u << floor_log2_u32(length);
  if ((index / 2) - 1 <= length - index) return index - 1;
  return length - index / 2;
}

/* A point record: dim coordinate words followed by the id word. */
typedef struct {
  uint32_t* w; /* n * (dim + 1) words */
  int dim;
  int stride;
} recs_t;

static inline float rec_coord(const recs_t* r, uint32_t i, int c) {
  float f;
  memcpy(&f, &r->w[(size_t)i * r->stride + c], 4);
  return f;
}
static inline uint32_t rec_id(const recs_t* r, uint32_t i) { return r->w[(size_t)i * r->stride + r->dim]; }

/* FKDTree_cpu.h:246-252: a < b on (coordinate c, id). */
static inline int rec_less(const recs_t* r, uint32_t a, uint32_t b, int c) {
  float fa = rec_coord(r, a, c), fb = rec_coord(r, b, c);
  if (fa == fb) return rec_id(r, a) < rec_id(r, b);
  return fa < fb;
}

static inline void rec_swap(recs_t* r, uint32_t a, uint32_t b) {
  if (a == b) return;
  uint32_t* pa = &r->w[(size_t)a * r->stride];
  uint32_t* pb = &r->w[(size_t)b * r->stride];
  for (int k = 0; k < r->stride; ++k) {
    uint32_t t = pa[k];
    pa[k] = pb[k];
    pb[k] = t;
  }
}

/* Places the k-th smallest (by rec_less on coordinate c) of [lo, lo+len) at
 * lo+k with smaller elements before it and larger ones after it: the contract
 * of std::nth_element as used at FKDTree_cpu.h:240-252. */
static void select_kth(recs_t* r, uint32_t lo, uint32_t k, uint32_t len, int c) {
  uint32_t left = lo, right = lo + len - 1, target = lo + k;
  uint64_t lcg = 0x2545F4914F6CDD1Dull ^ ((uint64_t)lo << 20) ^ len;
  while (right > left) {
    lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
    uint32_t p = left + (uint32_t)((lcg >> 33) % (uint64_t)(right - left + 1));
    rec_swap(r, p, right); /* pivot at right */
    uint32_t store = left;
    for (uint32_t i = left; i < right; ++i) {
      if (rec_less(r, i, right, c)) {
        rec_swap(r, i, store);
        ++store;
      }
    }
    rec_swap(r, store, right);
    if (store == target) return;
    if (store < target)
      left = store + 1;
    else
      right = store - 1;
  }
}

/* FKDTree_cpu.h:221-277.  coords_soa[c*n + i] and ids[i] describe the input
 * points; the result is written to tab_soa[c*n + i] / tab_ids[i] for heap
 * index i (FKDTree_cpu.h:323-326).  Returns 0, or -1 on bad arguments. */
int fkd_oracle_build(int dim, uint32_t n, const float* coords_soa, const uint32_t* ids, float* tab_soa,
                     uint32_t* tab_ids) {
  if (dim < 1 || dim > FKDO_MAXDIM) return -1;
  if (n == 0) return 0;
  recs_t r;
  r.dim = dim;
  r.stride = dim + 1;
  r.w = (uint32_t*)malloc((size_t)n * r.stride * 4);
  uint32_t* imin = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* ilen = (uint32_t*)malloc((size_t)n * 4);
  if (!r.w || !imin || !ilen) {
    free(r.w);
    free(imin);
    free(ilen);
    return -2;
  }
  for (uint32_t i = 0; i < n; ++i) {
    for (int c = 0; c < dim; ++c) memcpy(&r.w[(size_t)i * r.stride + c], &coords_soa[(size_t)c * n + i], 4);
    r.w[(size_t)i * r.stride + dim] = ids[i];
  }
  unsigned depth_max = floor_log2_u32(n);
  imin[0] = 0;
  ilen[0] = n;
  for (unsigned depth = 0; depth < depth_max; ++depth) {
    int c = (int)(depth % (unsigned)dim);
    uint32_t first = (1u << depth) - 1u;
    for (uint32_t j = 0; j < (1u << depth); ++j) {
      uint32_t i = first + j;
      uint32_t k = partition_complete(ilen[i]);
      select_kth(&r, imin[i], k, ilen[i], c);
      uint32_t src = imin[i] + k;
      for (int cc = 0; cc < dim; ++cc) tab_soa[(size_t)cc * n + i] = rec_coord(&r, src, cc);
      tab_ids[i] = rec_id(&r, src);
      uint32_t lson = 2 * i + 1, rson = lson + 1;
      if (lson < n) {
        imin[lson] = imin[i];
        ilen[lson] = k;
      }
      if (rson < n) {
        imin[rson] = imin[i] + k + 1;
        ilen[rson] = ilen[i] - 1 - k;
      }
    }
  }
  for (uint32_t i = (1u << depth_max) - 1u; i < n; ++i) {
    uint32_t src = imin[i];
    for (int cc = 0; cc < dim; ++cc) tab_soa[(size_t)cc * n + i] = rec_coord(&r, src, cc);
    tab_ids[i] = rec_id(&r, src);
  }
  free(r.w);
  free(imin);
  free(ilen);
  return 0;
}

/* The node intervals the reference build assigns (theIntervalMin/Length,
 * FKDTree_cpu.h:224-267), for checking a closed-form geometry against. */
int fkd_oracle_intervals(uint32_t n, uint32_t* imin, uint32_t* ilen) {
  if (n == 0) return 0;
  unsigned depth_max = floor_log2_u32(n);
  imin[0] = 0;
  ilen[0] = n;
  for (unsigned depth = 0; depth < depth_max; ++depth) {
    uint32_t first = (1u << depth) - 1u;
    for (uint32_t j = 0; j < (1u << depth); ++j) {
      uint32_t i = first + j;
      uint32_t k = partition_complete(ilen[i]);
      uint32_t lson = 2 * i + 1, rson = lson + 1;
      if (lson < n) {
        imin[lson] = imin[i];
        ilen[lson] = k;
      }
      if (rson < n) {
        imin[rson] = imin[i] + k + 1;
        ilen[rson] = ilen[i] - 1 - k;
      }
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ search */

typedef struct {
  int dim;
  uint32_t n;
  unsigned depth_max; /* theDepth */
  const float* tab;   /* tab[c*n + i] */
  const uint32_t* ids;
  float lo[FKDO_MAXDIM], hi[FKDO_MAXDIM];
} qctx_t;

/* FKDTree_cpu.h:302-308 */
static inline int intersects(const qctx_t* q, uint32_t i, int c) {
  float v = q->tab[(size_t)c * q->n + i];
  return v <= q->hi[c] && v >= q->lo[c];
}
/* FKDTree_cpu.h:310-321 */
static inline int in_box(const qctx_t* q, uint32_t i) {
  for (int c = 0; c < q->dim; ++c) {
    float v = q->tab[(size_t)c * q->n + i];
    if (!(v <= q->hi[c] && v >= q->lo[c])) return 0;
  }
  return 1;
}

typedef struct {
  uint32_t* buf;
  size_t cap;
  size_t len;
  uint32_t* out; /* NULL: count only */
  uint64_t count;
} emit_t;

static inline void emit(emit_t* e, uint32_t id) {
  if (e->out) e->out[e->count] = id;
  e->count++;
}

typedef struct {
  uint32_t* v;
  size_t cap, head, tail; /* [head, tail) live */
  size_t max_live;
} fifo_t;

static inline void fifo_push(fifo_t* f, uint32_t x) {
  if (f->tail == f->cap) {
    if (f->head > 0) {
      memmove(f->v, f->v + f->head, (f->tail - f->head) * 4);
      f->tail -= f->head;
      f->head = 0;
    }
    if (f->tail == f->cap) {
      f->cap = f->cap ? 2 * f->cap : 256;
      f->v = (uint32_t*)realloc(f->v, f->cap * 4);
    }
  }
  f->v[f->tail++] = x;
  size_t live = f->tail - f->head;
  if (live > f->max_live) f->max_live = live;
}

/* FKDTree_cpu.h:123-169: level-order frontier. */
static void search_level_order(const qctx_t* q, fifo_t* f, emit_t* e) {
  f->head = f->tail = 0;
  fifo_push(f, 0);
  for (unsigned depth = 0; depth < q->depth_max + 1; ++depth) {
    int c = (int)(depth % (unsigned)q->dim);
    size_t nthis = f->tail - f->head;
    for (size_t k = 0; k < nthis; ++k) {
      uint32_t i = f->v[f->head + k];
      int inter = intersects(q, i, c);
      if (inter && in_box(q, i)) emit(e, q->ids[i]);
      int lower = q->tab[(size_t)c * q->n + i] < q->lo[c];
      int start = lower, end = lower || inter;
      for (int s = start; s < end + 1; ++s) {
        uint32_t child = 2 * i + 1 + (uint32_t)s;
        if (child < q->n) fifo_push(f, child);
      }
    }
    f->head += nthis;
  }
}

/* FKDTree_cpu.h:72-121: pop-one BFS. */
static void search_bfs(const qctx_t* q, fifo_t* f, emit_t* e) {
  f->head = f->tail = 0;
  fifo_push(f, 0);
  while (f->tail > f->head) {
    uint32_t i = f->v[f->head++];
    int c = (int)(floor_log2_u32(i + 1) % (unsigned)q->dim);
    int inter = intersects(q, i, c);
    uint32_t first = 2 * i + 1;
    int maxsons = (first < q->n) + ((first + 1) < q->n);
    int nsons;
    if (inter) {
      if (in_box(q, i)) emit(e, q->ids[i]);
      nsons = maxsons;
    } else {
      int right_only = q->tab[(size_t)c * q->n + i] < q->lo[c];
      nsons = (right_only == maxsons) ? 0 : (maxsons < 1 ? maxsons : 1);
      first += (uint32_t)right_only;
    }
    for (int s = 0; s < nsons; ++s) fifo_push(f, first + (uint32_t)s);
  }
}

/* FKDTree_cpu.h:25-70: level order with arithmetic child selection.  Where
 * a node with only a left child misses the box and the walk turns right
 * (FKDTree_cpu.h:56-60), the reference pushes index n, one past the tables,
 * and reads theDimensions[c][n] at the next depth (undefined behaviour; it
 * emits nothing unless that stray value happens to lie in the box).  Here a
 * child index at or past n is never pushed. */
static void search_branchless(const qctx_t* q, fifo_t* f, emit_t* e) {
  f->head = f->tail = 0;
  fifo_push(f, 0);
  for (unsigned depth = 0; depth < q->depth_max + 1; ++depth) {
    int c = (int)(depth % (unsigned)q->dim);
    size_t nthis = f->tail - f->head;
    for (size_t k = 0; k < nthis; ++k) {
      uint32_t i = f->v[f->head + k];
      int inter = intersects(q, i, c);
      uint32_t first = 2 * i + 1;
      int maxsons = (first < q->n) + ((first + 1) < q->n);
      int nsons;
      if (inter) {
        if (in_box(q, i)) emit(e, q->ids[i]);
        nsons = maxsons;
      } else {
        nsons = maxsons < 1 ? maxsons : 1;
        first += (q->tab[(size_t)c * q->n + i] < q->lo[c]);
        if (first >= q->n) nsons = 0;
      }
      for (int s = 0; s < nsons; ++s) fifo_push(f, first + (uint32_t)s);
    }
    f->head += nthis;
  }
}

/* FKDTree_cpu.h:171-207: depth-first recursion. */
static void search_recursive(const qctx_t* q, emit_t* e, uint32_t i, int c) {
  uint32_t first = 2 * i + 1;
  int maxsons = (first < q->n) + ((first + 1) < q->n);
  int inter = intersects(q, i, c);
  int nsons;
  if (inter) {
    if (in_box(q, i)) emit(e, q->ids[i]);
    nsons = maxsons;
  } else {
    int lower = q->tab[(size_t)c * q->n + i] < q->lo[c];
    nsons = (lower && maxsons == 1) ? 0 : (maxsons < 1 ? maxsons : 1);
    first += (uint32_t)lower;
  }
  int cn = (c + 1) % q->dim;
  for (int s = 0; s < nsons; ++s) search_recursive(q, e, first + (uint32_t)s, cn);
}

/* FKDTree.h:54-86: a point is in the box iff every coordinate is inside the
 * closed interval; the scan runs over the table in heap order. */
static void search_brute(const qctx_t* q, emit_t* e) {
  for (uint32_t i = 0; i < q->n; ++i)
    if (in_box(q, i)) emit(e, q->ids[i]);
}

/* Runs `variant` (0 level order, 1 BFS, 2 branchless, 3 recursive, 4 brute
 * force) for nq boxes given as mins_soa[c*nq + j] / maxs_soa[c*nq + j].
 * counts[j] receives the number of results; when offsets and out are given,
 * the ids of box j are written to out[offsets[j] ...] in the order the
 * variant emits them.  max_frontier[j], when given, receives the largest
 * number of live frontier entries (variants 0-2). */
int fkd_oracle_search(int variant, int dim, uint32_t n, const float* tab_soa, const uint32_t* tab_ids, uint64_t nq,
                      const float* mins_soa, const float* maxs_soa, uint32_t* counts, uint32_t* max_frontier,
                      const uint64_t* offsets, uint32_t* out, int threads) {
  if (dim < 1 || dim > FKDO_MAXDIM || variant < 0 || variant > 4) return -1;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel
  {
    fifo_t f = {0};
#pragma omp for schedule(dynamic, 64)
    for (int64_t j = 0; j < (int64_t)nq; ++j) {
      qctx_t q;
      q.dim = dim;
      q.n = n;
      q.depth_max = floor_log2_u32(n);
      q.tab = tab_soa;
      q.ids = tab_ids;
      for (int c = 0; c < dim; ++c) {
        q.lo[c] = mins_soa[(size_t)c * nq + j];
        q.hi[c] = maxs_soa[(size_t)c * nq + j];
      }
      emit_t e = {0};
      e.out = (offsets && out) ? out + offsets[j] : NULL;
      f.max_live = 0;
      if (n > 0) {
        switch (variant) {
          case 0: search_level_order(&q, &f, &e); break;
          case 1: search_bfs(&q, &f, &e); break;
          case 2: search_branchless(&q, &f, &e); break;
          case 3: search_recursive(&q, &e, 0, 0); break;
          default: search_brute(&q, &e); break;
        }
      }
      counts[j] = (uint32_t)e.count;
      if (max_frontier) max_frontier[j] = (uint32_t)f.max_live;
    }
    free(f.v);
  }
  return 0;
}

/* Order-independent 64-bit digest of an id set: the wrap-around sum of a
 * 64-bit finaliser of every id.  Shared definition with the device code. */
static inline uint64_t fkd_mix64(uint32_t id) {
  uint64_t z = (uint64_t)id + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t fkd_oracle_mix64(uint32_t id) { return fkd_mix64(id); }

/* Per-box result count and digest with the recursive variant (which has no
 * capacity limit), for workloads whose result ids do not fit in memory. */
int fkd_oracle_search_digest(int dim, uint32_t n, const float* tab_soa, const uint32_t* tab_ids, uint64_t nq,
                             const float* mins_soa, const float* maxs_soa, uint32_t* counts, uint64_t* digests,
                             int threads) {
  if (dim < 1 || dim > FKDO_MAXDIM) return -1;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel
  {
    uint32_t* scratch = NULL;
    size_t cap = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t j = 0; j < (int64_t)nq; ++j) {
      qctx_t q;
      q.dim = dim;
      q.n = n;
      q.depth_max = floor_log2_u32(n);
      q.tab = tab_soa;
      q.ids = tab_ids;
      for (int c = 0; c < dim; ++c) {
        q.lo[c] = mins_soa[(size_t)c * nq + j];
        q.hi[c] = maxs_soa[(size_t)c * nq + j];
      }
      emit_t e = {0};
      if (n > 0) search_recursive(&q, &e, 0, 0); /* count */
      if (e.count > cap) {
        cap = e.count * 2;
        scratch = (uint32_t*)realloc(scratch, cap * 4);
      }
      emit_t w = {0};
      w.out = scratch;
      if (n > 0 && e.count) search_recursive(&q, &w, 0, 0);
      uint64_t d = 0;
      for (uint64_t k = 0; k < w.count; ++k) d += fkd_mix64(scratch[k]);
      counts[j] = (uint32_t)e.count;
      digests[j] = d;
    }
    free(scratch);
  }
  return 0;
}

/* Per-box digests of result lists already written out: box j's ids are
 * ids[offsets[j] .. offsets[j+1]).  Checks a search's output id for id
 * against fkd_oracle_search_digest / the reference's digests without
 * holding a second copy of the lists. */
int fkd_oracle_digest_lists(uint64_t nq, const uint64_t* offsets, const uint32_t* ids, uint64_t* digests,
                            int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t j = 0; j < (int64_t)nq; ++j) {
    uint64_t d = 0;
    for (uint64_t k = offsets[j]; k < offsets[j + 1]; ++k) d += fkd_mix64(ids[k]);
    digests[j] = d;
  }
  return 0;
}

/* Batched events: event e owns points [pt_off[e], pt_off[e+1]) of the
 * concatenated input and boxes [q_off[e], q_off[e+1]); each event is built and
 * searched independently (one OpenMP task per event, serial inside, the
 * structure of a per-event reference run).  dims[e] is the event's dimension;
 * coordinates of an event are stored SoA inside its own slice:
 * coords[base + c*n_e + i] with base = dim_off[e].  Outputs: the tables in the
 * same slice layout, and per box count + digest. */
int fkd_oracle_batch(uint32_t nev, const uint32_t* dims, const uint64_t* pt_off, const uint64_t* coord_off,
                     const float* coords, const uint32_t* ids, const uint64_t* q_off, const uint64_t* qcoord_off,
                     const float* mins, const float* maxs, float* tab, uint32_t* tab_ids, uint32_t* counts,
                     uint64_t* digests, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int64_t e = 0; e < (int64_t)nev; ++e) {
    uint32_t n = (uint32_t)(pt_off[e + 1] - pt_off[e]);
    int dim = (int)dims[e];
    const float* cs = coords + coord_off[e];
    float* ts = tab + coord_off[e];
    uint32_t* ti = tab_ids + pt_off[e];
    if (fkd_oracle_build(dim, n, cs, ids + pt_off[e], ts, ti) != 0) bad |= 1;
    uint64_t nq = q_off[e + 1] - q_off[e];
    if (fkd_oracle_search_digest(dim, n, ts, ti, nq, mins + qcoord_off[e], maxs + qcoord_off[e], counts + q_off[e],
                                 digests + q_off[e], 1) != 0)
      bad |= 1;
  }
  return bad ? -1 : 0;
}
