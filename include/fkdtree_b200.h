/*
 * fkdtree_b200.h -- C ABI of the B200 (sm_100a) FKDTree build and box search.
 *
 * The library (fkdtree_b200/libfkdtree_b200.so) builds the reference's flat,
 * heap-ordered kd-tree on the GPU and answers axis-aligned box queries on it.
 * The tree it builds is bit-identical to FKDTree_CPU::build
 * (FKDTree_cpu.h:221-277 of te42kyfo/FKDTree): node i holds one input point,
 * its split value is coordinate (depth(i) % dim) of that point, its children
 * are 2i+1 and 2i+2, and the tables returned by fkd_get_tables are exactly
 * theDimensions[d][i] / theIds[i] (FKDTree_cpu.h:323-326) -- provided the
 * input ids are unique (with repeated ids the order among points whose
 * split coordinate AND id tie is not defined by the reference either).
 *
 * Conventions
 *  - every entry point returns an fkd_status; 0 is success.  No exception or
 *    abort crosses the boundary.  fkd_last_error() describes the last failure
 *    of the calling thread.
 *  - coordinates are float32 and laid out SoA: coordinate c of point i is
 *    coords[c*n + i] (the layout of getDimensionVector, FKDTree_cpu.h:209-213,
 *    and of the OpenCL host upload, FKDTree_opencl.h:139-144).  Ids are uint32.
 *  - box j is [mins[c*q + j], maxs[c*q + j]] in every dimension c, bounds
 *    inclusive (FKDTree_cpu.h:302-321).
 *  - `mem` says where the caller's buffers live: FKD_MEM_HOST (pageable or
 *    pinned host memory; the call copies through the handle's device staging
 *    buffers and is synchronous) or FKD_MEM_DEVICE (device pointers on the
 *    handle's device; the call is stream-ordered on the handle's stream and,
 *    unless the handle was created with FKD_FLAG_ASYNC, synchronises before it
 *    returns so that errors can be reported).
 *  - a handle is bound to one device and one stream.  Once a build has
 *    returned, searches (fkd_search*, fkd_search_radius*, fkd_search_knn,
 *    fkd_get_tables) may be called on the handle from any number of host
 *    threads at once, as the reference's searches are (main.cpp:351-359):
 *    each call leases its own scratch from the handle.  Host-memory calls run
 *    on a stream of that scratch (concurrent calls overlap on the GPU, each
 *    ordered after the last build); device-memory calls run on the handle's
 *    stream.  A build, fkd_set_param, fkd_set_mlp, fkd_set_stream or
 *    fkd_sync must not overlap any other call on the same handle, and with
 *    FKD_FLAG_ASYNC the caller orders its calls.  Different handles are
 *    independent.
 *  - NaN coordinates are rejected (FKD_ERR_NAN): the reference comparator
 *    (FKDTree_cpu.h:246-252) is not a strict weak order with NaN.  -0.0 and
 *    +0.0 compare equal and tie on id, as in the reference.
 *  - returned result ids are the tree's id values (theIds, FKDTree_cpu.h:148),
 *    not array positions.
 */
#ifndef FKDTREE_B200_H_
#define FKDTREE_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FKD_API __attribute__((visibility("default")))
#else
#define FKD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fkd_status {
  FKD_OK = 0,
  FKD_ERR_ARG = 1,       /* bad argument (null pointer, unsupported dim, size) */
  FKD_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  FKD_ERR_NOMEM = 3,     /* device or pinned allocation failed */
  FKD_ERR_NAN = 4,       /* a coordinate is NaN */
  FKD_ERR_STATE = 5,     /* e.g. search before build */
  FKD_ERR_CAPACITY = 6,  /* a result or frontier bound was exceeded; nothing was silently dropped */
  FKD_ERR_INTERNAL = 7,  /* a device-side consistency check failed */
  FKD_ERR_TIMEOUT = 8    /* reserved for a bounded device-side wait that gives up; no kernel of
                            this version waits on another, so no call returns it today */
} fkd_status;

enum { FKD_MEM_HOST = 0, FKD_MEM_DEVICE = 1 };

/* fkd_create flags */
enum {
  FKD_FLAG_ASYNC = 1u << 0 /* device-memory calls return without synchronising;
                              errors are reported by fkd_sync */
};

typedef struct fkd_tree_s* fkd_tree;

/* Version string of the library. */
FKD_API const char* fkd_version(void);

/* Number of CUDA kernels this library has launched in this process (all
 * handles, all threads).  Telemetry for benchmarks; no reference counterpart. */
FKD_API uint64_t fkd_kernel_launches(void);

/* Description of the last failure on the calling thread ("" if none). */
FKD_API const char* fkd_last_error(void);

/* Test hook (no reference counterpart): the device allocation `after`
 * allocations from now -- by any tree or batch handle of this process --
 * fails as if the device were out of memory, so callers can test their
 * FKD_ERR_NOMEM paths; -1 turns it off (the default).  The failing call
 * returns FKD_ERR_NOMEM and the handle stays usable. */
FKD_API void fkd_debug_fail_alloc(int32_t after);

/* Creates an empty tree for points of `dim` coordinates (1..4) on the current
 * CUDA device.  Replaces the FKDTree_CPU constructor (FKDTree_cpu.h:19-23);
 * the points are passed to fkd_build instead.  `stream` is a cudaStream_t
 * (NULL = the legacy default stream). */
FKD_API fkd_status fkd_create(int dim, uint32_t flags, void* stream, fkd_tree* out);
FKD_API fkd_status fkd_destroy(fkd_tree h);
FKD_API fkd_status fkd_set_stream(fkd_tree h, void* stream);

/* Builds the tree over n points.  Replaces FKDTree_CPU::build
 * (FKDTree_cpu.h:221-277) together with the point copy of its constructor.
 * coords: dim*n floats SoA; ids: n uint32.  n may be 0 (empty tree).  The
 * library keeps its own copy; the caller's buffers may be reused on return
 * (for FKD_MEM_DEVICE with FKD_FLAG_ASYNC: once the stream has passed the
 * call). */
FKD_API fkd_status fkd_build(fkd_tree h, const float* coords, const uint32_t* ids, uint64_t n, int mem);

/* Same as fkd_build, from points in the reference's FKDPoint<float, dim>
 * layout (FKDPoint.h:102-103, the element type of the std::vector the
 * FKDTree_CPU constructor takes, FKDTree_cpu.h:19-23): per point dim floats
 * then the uint32 id, (dim + 1) * 4 bytes, n points back to back.  Saves the
 * caller the conversion to SoA; the tree is the same. */
FKD_API fkd_status fkd_build_points(fkd_tree h, const void* points, uint64_t n, int mem);

/* Builds one small tree without allocating any memory (no counterpart in the
 * reference).  For callers that may not call cudaMalloc / cudaFree while
 * they work -- code inside a framework that owns all device memory through
 * its own pool, where those calls would synchronise the device or could fail
 * mid-event.  All buffers are the caller's device memory: coords (dim*n SoA),
 * ids (n) in; tab (dim*n SoA, theDimensions) and tab_ids (n, theIds) out, the
 * same tables fkd_build + fkd_get_tables produce.  The library works in a
 * fixed scratch array of its own (one per device, kept until exit), so n is
 * limited to fkd_build_noalloc_max_points(dim) (4096, or 3072 for dim 4);
 * larger n is rejected with FKD_ERR_ARG.  The first call on a device looks up
 * the scratch address and keeps it for the life of the process -- make it
 * before any stream capture; a cudaDeviceReset after that first call is not
 * supported (the kept address would belong to the destroyed context).  Calls share the
 * scratch: calls whose GPU work overlaps (other streams or threads on the same
 * device) race and must be serialised by the caller.  Synchronises `stream`
 * before returning, to report device-side errors. */
FKD_API fkd_status fkd_build_noalloc(int dim, const float* coords, const uint32_t* ids, uint32_t n, float* tab,
                                     uint32_t* tab_ids, void* stream);
FKD_API uint32_t fkd_build_noalloc_max_points(int dim);

/* Number of points of the last build. */
FKD_API fkd_status fkd_size(fkd_tree h, uint64_t* n);

/* Copies the tables out: tab[c*n + i] = theDimensions[c][i], tab_ids[i] =
 * theIds[i].  Replaces getDimensionVector / getIdVector
 * (FKDTree_cpu.h:209-213; the OpenCL backend's lazy download,
 * FKDTree_opencl.h:194-206).  Either pointer may be NULL. */
FKD_API fkd_status fkd_get_tables(fkd_tree h, float* tab, uint32_t* tab_ids, int mem);

/* Result count of every box (pass 1 of the two-pass search).  Replaces the
 * per-box counts of FKDTree_OpenCL::search_in_the_box_multiple
 * (FKDTree_opencl.h:123-164) and the counting half of CUDAKernelWrapper
 * (searchInTheBoxCuda.cu:174-185, main.cpp:305). */
FKD_API fkd_status fkd_search_count(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint32_t* counts,
                            int mem);

/* Writes the ids of box j to ids_out[offsets[j] .. offsets[j] + count_j)
 * (pass 2).  offsets has q+1 entries (exclusive prefix sum of the counts of
 * fkd_search_count, offsets[q] = total); ids_out holds offsets[q] ids.
 * Within a box the ids come in ascending heap-index order, the order
 * search_in_the_box / _BFS / _branchless emit them (FKDTree_cpu.h:123-169,
 * 72-121, 25-70), when `ordered` is nonzero; otherwise in traversal order. */
FKD_API fkd_status fkd_search_write(fkd_tree h, const float* mins, const float* maxs, uint64_t q, const uint64_t* offsets,
                            uint32_t* ids_out, int ordered, int mem);

/* Count, prefix sum and write in one call.  offsets_out receives q+1 entries;
 * at most `capacity` ids are written; *total receives the number of results.
 * Returns FKD_ERR_CAPACITY (and writes no ids) when total > capacity.
 * Replaces search_in_the_box applied to a batch of boxes
 * (FKDTree_cpu.h:123-169 under main.cpp:369-381) and the stub
 * search_in_the_box_multiple (FKDTree_cpu.h:215-219). */
FKD_API fkd_status fkd_search(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint64_t* offsets_out,
                      uint32_t* ids_out, uint64_t capacity, uint64_t* total, int ordered, int mem);

/* Per-box count and order-independent 64-bit digest of the id set (the
 * wrap-around sum of a 64-bit finaliser of every id), for workloads whose
 * result ids do not fit in memory.  No reference counterpart; it stands in
 * for test_correct_search (FKDTree.h:54-86) at scale. */
FKD_API fkd_status fkd_search_digest(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint32_t* counts,
                             uint64_t* digests, int mem);

/* ------------------------------------------------ radius and kNN search
 * No reference counterpart (the reference answers boxes only); both walk the
 * same tree with the reference's split rule (FKDTree_cpu.h:240-269) and
 * prune by the distance to the split plane, exactly (no point is missed).
 * centers: dim*q floats SoA like the boxes.  Distances are squared Euclidean
 * in float32, evaluated as (((0 + (p0-c0)^2) + (p1-c1)^2) + ...) with every
 * operation rounded separately (no fused multiply-add). */

/* Number of points within distance radii[j] of centre j: those with
 * d2 <= radii[j]*radii[j] (rounded to float).  A negative or NaN radius, or a
 * centre with a NaN coordinate, matches nothing. */
FKD_API fkd_status fkd_search_radius_count(fkd_tree h, const float* centers, const float* radii, uint64_t q,
                                           uint32_t* counts, int mem);
/* Ids of those points, query j in ids_out[offsets_out[j] .. offsets_out[j+1]):
 * in ascending heap-index order when `ordered` is nonzero, otherwise in the
 * walk's depth-first order (deterministic; the same set).  offsets_out
 * receives q+1 entries, *total the number of results; FKD_ERR_CAPACITY (no
 * ids written) when total > capacity. */
FKD_API fkd_status fkd_search_radius(fkd_tree h, const float* centers, const float* radii, uint64_t q,
                                     uint64_t* offsets_out, uint32_t* ids_out, uint64_t capacity, uint64_t* total,
                                     int ordered, int mem);
/* The k nearest points of every centre (1 <= k <= fkd_knn_max_k()), ascending
 * in (d2, id): ids_out[j*k + m] and, unless dist2_out is NULL,
 * dist2_out[j*k + m] = d2.  Ties of d2 go to the smaller id, so the answer
 * depends on the point set only.  Points with a NaN d2 never qualify; rows
 * with fewer than k neighbours end in id 0xffffffff, d2 = +inf. */
FKD_API fkd_status fkd_search_knn(fkd_tree h, const float* centers, uint64_t q, uint32_t k, uint32_t* ids_out,
                                  float* dist2_out, int mem);
FKD_API uint32_t fkd_knn_max_k(void);

/* Waits for the handle's stream and reports any device-side error latched by
 * earlier asynchronous calls. */
FKD_API fkd_status fkd_sync(fkd_tree h);

/* Tuning knobs of one tree, same names and ranges as fkd_batch_set_param
 * ("hist_ctas" takes effect at the next build; "search_lanes" applies to
 * fkd_search_count / fkd_search_digest), plus
 *   "box_order"     (0/1, default 1): searches visit the boxes in the spatial
 *                   order of their centres (tree cell), not in input order
 *   "small_select"  (0/1, default 1): global levels whose segments are small
 *                   select each segment with one CTA in shared memory
 *   "search_record" (0/1, default 1): fkd_search's count pass records every
 *                   box's result so that the write needs no second traversal
 *   "search_one"    (0/1, default 1): fkd_search of a single host-memory box
 *                   runs one warp over the tree level by level (the level-order
 *                   list straight away, one launch and one wait); boxes with a
 *                   NaN bound, very wide frontiers or more than 65,536 results
 *                   take the general count + write path
 *   "search_pool"   entries of the record pools (0, the default: sized by the
 *                   previous call's demand; boxes that do not fit are traversed
 *                   again, so any size gives the same results)
 *   "search_bucket" (0..6, default 5): box searches scan the visited subtrees
 *                   of height <= this many levels (at most 2^(v+1)-1 points)
 *                   point by point in in-order layout instead of walking them;
 *                   0 walks every level.  Costs 16 bytes per point of device
 *                   memory for the in-order copy of the nodes.
 *   "bucket_runs"   (0/1, default 1): unordered fkd_search records the leaf
 *                   buckets' hits at consecutive in-order positions as runs
 *                   (0: every hit as a single id)
 *   "search_bucket_lanes" (0..3, default 0): the same for the count / digest
 *                   searches with fewer than 32 lanes per box ("search_lanes"):
 *                   one lane scans a visited subtree of at most 2^(v+1)-1 points
 *   "small_fix"     (0/1, default 1): a global level's select stops once at
 *                   most 32 candidates are left; the partition parks them and
 *                   one warp orders them by (coordinate, id), instead of more
 *                   digit passes
 *   "subtree_size"  (0, 512 or 1024; 0 = 1024): the largest subtree the
 *                   presorted-list kernel (dims 1-3) finishes in shared memory;
 *                   smaller subtrees take one more global level.  Re-plans at
 *                   the next build.
 *   "lin_pass"      (0/1, default 1): a segment's first digit pass bins its
 *                   value range (known from its parent's partition) in 2048
 *                   equal float intervals rather than by the top key bits
 *   "kernel_events" (0/1): record CUDA events around the kernels of every
 *                   fkd_build and fkd_search call for fkd_kernel_times (only
 *                   calls on the handle's stream, from one thread).
 * No reference counterpart. */
FKD_API fkd_status fkd_set_param(fkd_tree h, const char* name, int64_t value);
/* Device times (ms) of the kernels of the build / search `back` calls ago
 * (0 = the last; at most 63), measured by CUDA events on the handle's stream:
 * ms[0] count pass, ms[1] write pass (fkd_search), ms[2] whole build,
 * ms[3] global levels, ms[4] shared-memory subtree kernel (fkd_build).
 * Requires "kernel_events" = 1.  No reference counterpart. */
FKD_API fkd_status fkd_kernel_times(fkd_tree h, uint32_t back, float* ms);

/* ---------------------------------------------------------------- batches
 * Many independent events (one tree each) built and searched together.  No
 * reference counterpart: the reference constructs one FKDTree_CPU per event
 * (FKDTree_cpu.h:19-23) and calls build() (:221-277) and search_in_the_box
 * (:123-169) on each.
 *
 * Layout: event e owns points [pt_off[e], pt_off[e+1]) and boxes
 * [q_off[e], q_off[e+1]) of the concatenated id / count / digest arrays; its
 * coordinates form their own SoA slice of the concatenated coordinate array:
 * coordinate c of its point i is coords[coff(e) + c*n_e + i] with
 * coff(e) = sum over e' < e of dims[e'] * n_e' (boxes likewise with q_e).
 * Events may mix dimensions (1..4). */
typedef struct fkd_batch_s* fkd_batch;

/* Plans the batch from its sizes (the plan is reused by every later call). */
FKD_API fkd_status fkd_batch_create(uint32_t n_events, const uint32_t* dims, const uint64_t* pt_off,
                                    const uint64_t* q_off, uint32_t flags, void* stream, fkd_batch* out);
FKD_API fkd_status fkd_batch_destroy(fkd_batch b);
/* Tuning knobs used by the autotuner (fkdtree_b200/autotune.py):
 *   "hist_ctas"    digit-pass CTAs per level (0 = four per SM); re-plans the batch
 *   "search_lanes" lanes per box of the count / digest search: 1, 2, 4, 8, 16
 *                  or 32 (0 = 32, one warp per box)
 *   "search_big_n", "search_lanes_big"  digest search: events of at least
 *                  search_big_n points search with search_lanes_big lanes per
 *                  box in a launch of their own (0: one launch for all)
 *   "subtree"      shared-memory subtree kernel: 0 auto (presorted lists for
 *                  dims 1-3, radix select for dim 4), 1 radix select, 2 lists
 *   "small_fix", "lin_pass", "search_bucket", "search_bucket_lanes",
 *   "subtree_size"  as fkd_set_param's
 *                  ("subtree_size" re-plans the batch)
 * A failed "hist_ctas" re-plan leaves the batch without a plan: builds then
 * return FKD_ERR_STATE until a re-plan succeeds.
 * No reference counterpart (the reference has one fixed launch shape). */
FKD_API fkd_status fkd_batch_set_param(fkd_batch b, const char* name, int64_t value);
/* Builds every event; the tables equal one FKDTree_CPU::build per event. */
FKD_API fkd_status fkd_batch_build(fkd_batch b, const float* coords, const uint32_t* ids, int mem);
/* Tables of every event in the coordinate / id layout above. */
FKD_API fkd_status fkd_batch_get_tables(fkd_batch b, float* tab, uint32_t* tab_ids, int mem);
/* Per-box result count and order-independent digest (see fkd_search_digest);
 * each box searches its own event's tree. */
FKD_API fkd_status fkd_batch_search_digest(fkd_batch b, const float* mins, const float* maxs, uint32_t* counts,
                                           uint64_t* digests, int mem);
/* Build + digest search of device buffers as ONE CUDA graph launch; the graph
 * is captured on the first call and replayed while the buffers stay the same.
 * The batch's stream must not be the legacy default stream (a NULL stream at
 * fkd_batch_create gives the batch its own stream). */
FKD_API fkd_status fkd_batch_run(fkd_batch b, const float* coords, const uint32_t* ids, const float* mins,
                                 const float* maxs, uint32_t* counts, uint64_t* digests);
FKD_API fkd_status fkd_batch_sync(fkd_batch b);

/* -------------------------------------------------------- learned split
 * A 40 -> 64 -> 64 -> 1 MLP (GELU, bf16 operands, fp32 accumulation) that
 * predicts where a node's split value lies, from cheap summaries of the node:
 * the bounding box of a 256-point sample (6 floats), log2 of the point count,
 * the depth and a 32-bin histogram of the sample along the split dimension
 * (FKD_MLP_IN = 40 features, layout in fkd_features.cu).  The prediction only
 * chooses where the exact radix select starts; a verifying count decides
 * whether it holds and the plain select runs when it does not, so the tree is
 * bit-identical either way.  No reference counterpart.
 *
 * Parameters (fkd_mlp_param_count() floats): W1[48][64] (rows 40..47 zero),
 * b1[64], W2[64][64], b2[64], w3[64], b3. */
#define FKD_MLP_IN 40
typedef struct fkd_mlp_s* fkd_mlp;

FKD_API fkd_status fkd_mlp_create(uint32_t seed, fkd_mlp* out);
FKD_API fkd_status fkd_mlp_destroy(fkd_mlp m);
FKD_API uint64_t fkd_mlp_param_count(void);
FKD_API fkd_status fkd_mlp_get_params(fkd_mlp m, float* params);
FKD_API fkd_status fkd_mlp_set_params(fkd_mlp m, const float* params);
/* y[i] = MLP(x[i*40 .. i*40+39]) */
FKD_API fkd_status fkd_mlp_forward(fkd_mlp m, const float* x, uint64_t n, float* y, int mem);
/* Gradient of mean((y - t)^2)/2 w.r.t. every parameter (host output). */
FKD_API fkd_status fkd_mlp_grad(fkd_mlp m, const float* x, const float* t, uint64_t n, float* grad, float* loss,
                                int mem);
/* Adam training on the GPU; losses[epoch] receives the mean batch loss. */
FKD_API fkd_status fkd_mlp_train(fkd_mlp m, const float* x, const float* t, uint64_t n, uint32_t epochs,
                                 uint32_t batch, float lr, uint32_t seed, float* losses, int mem);
/* Learned split for later builds of a tree / batch (m NULL: plain radix
 * select).  delta is the bracket half-width in units of the node's sample
 * range along the split dimension.  The model must outlive its use. */
FKD_API fkd_status fkd_set_mlp(fkd_tree h, fkd_mlp m, float delta);
FKD_API fkd_status fkd_batch_set_mlp(fkd_batch b, fkd_mlp m, float delta);
/* stats[0] brackets predicted, [1] verified (the select started inside the
 * predicted block), [2] fell back to the plain select, [3] digit passes run
 * over a segment by the global levels' selects (with or without a network:
 * what a verified bracket saves shows as fewer passes); cumulative until
 * reset. */
FKD_API fkd_status fkd_learn_stats(fkd_tree h, uint64_t* stats, int reset);
FKD_API fkd_status fkd_batch_learn_stats(fkd_batch b, uint64_t* stats, int reset);
/* Exact (plain) build of a batch that also records, for every node the
 * global kernels split, its features and target (the split value's position
 * in the node's sample range): training data for the learned split.  At most
 * cap rows are written (host arrays x_out: cap*40, t_out: cap); *n_out
 * receives the number of recorded nodes. */
FKD_API fkd_status fkd_batch_record(fkd_batch b, const float* coords, const uint32_t* ids, float* x_out,
                                    float* t_out, uint64_t cap, uint64_t* n_out, int mem);

#ifdef __cplusplus
}
#endif

#endif /* FKDTREE_B200_H_ */
