// Drop-in check: the reference's own FKDTree_CPU and FKDTree_CUDA side by side
// behind the reference's FKDTree<T, dim> interface.  Built by oracle/Makefile
// (target `dropin`, against the reference headers) into oracle/_ref/test_dropin;
// run on a GPU by tests/test_dropin_gpu.py.  Prints "DROPIN OK" on success.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "FKDTree_CUDA.h"
#include "FKDTree_cpu.h"

// squared distance as the library evaluates it: each operation rounded on its
// own, coordinates in order (the Makefile compiles this with -ffp-contract=off)
template <int D>
static float dist2(const FKDPoint<float, D>& p, const FKDPoint<float, D>& c) {
  float acc = 0.f;
  for (int d = 0; d < D; ++d) {
    const float t = p[d] - c[d];
    acc = acc + t * t;
  }
  return acc;
}

template <unsigned D>
static int run(unsigned n, unsigned seed, float hw) {
  std::mt19937 gen(seed);
  std::uniform_real_distribution<float> u(0.f, 1.f);
  std::vector<FKDPoint<float, D>> pts(n), lo(n), hi(n);
  for (unsigned i = 0; i < n; ++i) {
    for (unsigned c = 0; c < D; ++c) {
      float x = u(gen);
      if (c == 3) x = (float)(int)(x * 16) / 16.f;  // a discrete fourth coordinate: heavy ties
      pts[i].setDimension(c, x);
      lo[i].setDimension(c, x - hw);
      hi[i].setDimension(c, x + hw);
    }
    pts[i].setId(i);
  }
  FKDTree_CPU<float, D> cpu(pts);
  cpu.build();
  std::unique_ptr<FKDTree<float, D>> gpu(new FKDTree_CUDA<float, D>(pts));
  gpu->build();
  for (unsigned c = 0; c < D; ++c)
    if (gpu->getDimensionVector(c) != cpu.getDimensionVector(c)) {
      std::printf("dim %u: theDimensions differ\n", c);
      return 1;
    }
  if (gpu->getIdVector() != cpu.getIdVector()) {
    std::printf("theIds differ\n");
    return 1;
  }
  if (!gpu->test_correct_build()) {
    std::printf("test_correct_build failed\n");
    return 1;
  }
  const unsigned q = n < 2000 ? n : 2000;
  std::vector<unsigned> counts = gpu->search_in_the_box_multiple(
      std::vector<FKDPoint<float, D>>(lo.begin(), lo.begin() + q), std::vector<FKDPoint<float, D>>(hi.begin(), hi.begin() + q));
  auto* cu = static_cast<FKDTree_CUDA<float, D>*>(gpu.get());
  std::vector<uint64_t> offs;
  std::vector<unsigned> ids;
  cu->search_in_the_box_batch(std::vector<FKDPoint<float, D>>(lo.begin(), lo.begin() + q),
                              std::vector<FKDPoint<float, D>>(hi.begin(), hi.begin() + q), offs, ids, true);
  for (unsigned j = 0; j < q; ++j) {
    std::vector<unsigned> want = cpu.search_in_the_box(lo[j], hi[j]);  // the reference's order
    std::vector<unsigned> got = gpu->search_in_the_box(lo[j], hi[j]);
    std::vector<unsigned> batch(ids.begin() + offs[j], ids.begin() + offs[j + 1]);
    if (got != want || batch != want || counts[j] != want.size()) {
      std::printf("box %u: results differ (%zu vs %zu)\n", j, got.size(), want.size());
      return 1;
    }
    if (j < 50 && !test_correct_search(pts, got, lo[j], hi[j])) {
      std::printf("box %u: test_correct_search failed\n", j);
      return 1;
    }
  }
  // radius and kNN queries against the reference's box search and a brute force
  std::vector<unsigned> heap_of(n);  // id -> heap index
  for (unsigned i = 0; i < n; ++i) heap_of[cpu.getIdVector()[i]] = i;
  for (unsigned j = 0; j < 200 && j < n; ++j) {
    const float r = hw * (1.f + (float)(j % 3));
    FKDPoint<float, D> blo, bhi;
    for (unsigned c = 0; c < D; ++c) {
      blo.setDimension(c, pts[j][c] - r * 1.001f - 1e-6f);
      bhi.setDimension(c, pts[j][c] + r * 1.001f + 1e-6f);
    }
    std::vector<unsigned> box, want;
    cpu.search_in_the_box_recursive(blo, bhi, box);  // no frontier bound
    for (unsigned id : box)
      if (dist2(pts[id], pts[j]) <= r * r) want.push_back(id);
    std::sort(want.begin(), want.end(), [&](unsigned a, unsigned b) { return heap_of[a] < heap_of[b]; });
    if (cu->search_in_the_ball(pts[j], r) != want) {
      std::printf("ball %u: results differ\n", j);
      return 1;
    }
    std::vector<std::pair<float, unsigned>> all;
    for (unsigned i = 0; i < n; ++i) all.emplace_back(dist2(pts[i], pts[j]), pts[i].getId());
    const unsigned k = 1 + j % 20;
    std::partial_sort(all.begin(), all.begin() + k, all.end());
    std::vector<float> d2;
    std::vector<unsigned> nn = cu->nearest_neighbours(pts[j], k, &d2);
    for (unsigned m = 0; m < k; ++m)
      if (nn.size() != k || nn[m] != all[m].second || d2[m] != all[m].first) {
        std::printf("knn %u: results differ at %u\n", j, m);
        return 1;
      }
  }
  std::printf("dim %u n %u: %u boxes identical, 200 balls and kNN rows identical\n", D, n, q);
  return 0;
}

// main.cpp:351-359's pattern: one built tree, `threads` host threads each
// calling search_in_the_box on its own slice of the boxes at the same time,
// every list compared with the reference's; then the single-box latency of
// one thread alone and the box rate of all threads.
static int run_threads(unsigned n, unsigned q, unsigned threads, float hw) {
  std::mt19937 gen(7);
  std::uniform_real_distribution<float> u(0.f, 1.f);
  std::vector<FKDPoint<float, 3>> pts(n), lo(q), hi(q);
  for (unsigned i = 0; i < n; ++i) {
    for (unsigned c = 0; c < 3; ++c) pts[i].setDimension(c, u(gen));
    pts[i].setId(i);
  }
  for (unsigned j = 0; j < q; ++j)
    for (unsigned c = 0; c < 3; ++c) {
      lo[j].setDimension(c, pts[j % n][c] - hw);
      hi[j].setDimension(c, pts[j % n][c] + hw);
    }
  FKDTree_CPU<float, 3> cpu(pts);
  cpu.build();
  std::unique_ptr<FKDTree<float, 3>> gpu(new FKDTree_CUDA<float, 3>(pts));
  gpu->build();
  std::vector<std::vector<unsigned>> got(q);
  std::atomic<int> failures(0);
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&, t]() {
      try {
        for (unsigned j = t; j < q; j += threads) got[j] = gpu->search_in_the_box(lo[j], hi[j]);
      } catch (const std::exception& e) {
        std::printf("thread %u: %s\n", t, e.what());
        failures++;
      }
    });
  for (auto& th : pool) th.join();
  auto t1 = std::chrono::steady_clock::now();
  if (failures) return 1;
  for (unsigned j = 0; j < q; ++j)
    if (got[j] != cpu.search_in_the_box(lo[j], hi[j])) {
      std::printf("threads: box %u differs\n", j);
      return 1;
    }
  const unsigned q1 = std::min(q, 2000u);
  auto t2 = std::chrono::steady_clock::now();
  for (unsigned j = 0; j < q1; ++j)
    if (gpu->search_in_the_box(lo[j], hi[j]).size() != got[j].size()) return 1;
  auto t3 = std::chrono::steady_clock::now();
  const double mt = std::chrono::duration<double>(t1 - t0).count();
  const double st = std::chrono::duration<double>(t3 - t2).count();
  std::printf("threads %u: %u boxes identical to FKDTree_CPU\n", threads, q);
  std::printf("LATENCY {\"single_box_us\": %.2f, \"threads\": %u, \"boxes_per_s_threaded\": %.1f, \"n\": %u}\n",
              1e6 * st / q1, threads, q / mt, n);
  return 0;
}

int main() {
  int rc = 0;
  rc |= run<3>(50000, 1, 0.02f);
  rc |= run<4>(30000, 2, 0.05f);
  rc |= run<2>(7777, 3, 0.01f);
  rc |= run_threads(100000, 20000, 8, 0.01f);
  if (rc == 0) std::printf("DROPIN OK\n");
  return rc;
}
