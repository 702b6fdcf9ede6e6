// FKDTree_CUDA.h -- drop-in replacement for the reference's FKDTree_CPU<TYPE, dim>
// backed by the B200 library (include/fkdtree_b200.h).
//
// Usage is the reference's (main.cpp:203-205, :351-375):
//
//     #include "FKDTree_CUDA.h"          // needs FKDPoint.h / FKDTree.h on the include path
//     std::unique_ptr<FKDTree<float, 3>> t(new FKDTree_CUDA<float, 3>(points));
//     t->build();
//     std::vector<unsigned int> ids = t->search_in_the_box(minPoint, maxPoint);
//
// It derives from the reference's abstract FKDTree<TYPE, dim> (FKDTree.h:6-22),
// so code written against that interface -- including its test_correct_build
// and test_correct_search helpers -- runs unchanged.  Semantics:
//   * build() produces the reference's tables bit for bit (unique ids);
//   * search_in_the_box / _BFS / _branchless return the reference's list in the
//     reference's order (ascending heap index, FKDTree_cpu.h:123-169, 72-121,
//     25-70); search_in_the_box_recursive appends the same set to foundPoints
//     (in ascending heap order rather than the reference's depth-first order);
//   * search_in_the_box_multiple returns per-box counts, the OpenCL backend's
//     meaning (FKDTree_opencl.h:123-164) -- the CPU backend's is a stub;
//   * search_in_the_box_batch is the bulk form (one GPU launch for all boxes);
//   * search_in_the_ball / nearest_neighbours add radius and kNN queries on the
//     same tree (no reference counterpart; fkd_search_radius, fkd_search_knn);
//   * getDimensionVector / getIdVector download the tables lazily after a
//     build, like FKDTree_OpenCL (FKDTree_opencl.h:194-206);
//   * failures throw std::runtime_error carrying fkd_last_error(); the
//     reference aborts or prints instead.
// Threads: as with the reference, once build() has returned any number of
// threads may search one tree at the same time (main.cpp:351-359 runs
// search_in_the_box from a TBB parallel_for); every search call leases its own
// scratch and stream inside the library.  build() must not overlap any other
// call on the same tree.  A single-box search is a host round trip to the GPU
// (tens of microseconds); callers with many boxes should use
// search_in_the_box_batch, one launch for all of them.
#ifndef FKDTREE_CUDA_H_
#define FKDTREE_CUDA_H_

#include <algorithm>  // FKDTree.h uses std::find without including it
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "FKDPoint.h"
#include "FKDTree.h"
#include "fkdtree_b200.h"

template <class TYPE, unsigned int numberOfDimensions>
class FKDTree_CUDA : public FKDTree<TYPE, numberOfDimensions> {
  static_assert(std::is_same<TYPE, float>::value, "the B200 tree stores float32 coordinates");
  static_assert(numberOfDimensions >= 1 && numberOfDimensions <= 4, "1 to 4 dimensions");

 public:
  typedef FKDPoint<TYPE, numberOfDimensions> Point;

  // The points are kept as given (the reference copies them into its own SoA
  // arrays, FKDTree_cpu.h:19-23); build() uploads them in FKDPoint layout.
  explicit FKDTree_CUDA(const std::vector<Point>& points, void* stream = nullptr)
      : n_(points.size()), points_(points), synced_(false) {
    static_assert(sizeof(Point) == (numberOfDimensions + 1) * sizeof(float),
                  "FKDPoint<float, dim> is dim floats followed by the id (FKDPoint.h:102-103)");
    check(fkd_create((int)numberOfDimensions, 0u, stream, &h_));
  }

  ~FKDTree_CUDA() { fkd_destroy(h_); }
  FKDTree_CUDA(const FKDTree_CUDA&) = delete;
  FKDTree_CUDA& operator=(const FKDTree_CUDA&) = delete;

  void build() override {
    check(fkd_build_points(h_, points_.data(), n_, FKD_MEM_HOST));
    std::lock_guard<std::mutex> g(tables_mu_);
    synced_ = false;
  }

  // Ids of the points within `radius` of `centre` (squared float32 distance
  // <= radius * radius), ascending heap order.  No reference counterpart.
  std::vector<unsigned int> search_in_the_ball(const Point& centre, float radius) {
    float c[numberOfDimensions];
    for (unsigned int d = 0; d < numberOfDimensions; ++d) c[d] = centre[d];
    thread_local std::vector<unsigned int> buf(256);
    uint64_t offsets[2] = {0, 0};
    uint64_t total = 0;
    fkd_status s = fkd_search_radius(h_, c, &radius, 1, offsets, buf.data(), buf.size(), &total, 1, FKD_MEM_HOST);
    if (s == FKD_ERR_CAPACITY && total > buf.size()) {
      buf.resize(total + total / 2);
      s = fkd_search_radius(h_, c, &radius, 1, offsets, buf.data(), buf.size(), &total, 1, FKD_MEM_HOST);
    }
    check(s);
    return std::vector<unsigned int>(buf.begin(), buf.begin() + total);
  }

  // The k nearest points of `centre`, ascending in (squared distance, id);
  // fewer than k when the tree is smaller.  No reference counterpart.
  std::vector<unsigned int> nearest_neighbours(const Point& centre, unsigned int k,
                                               std::vector<float>* dist2 = nullptr) {
    float c[numberOfDimensions];
    for (unsigned int d = 0; d < numberOfDimensions; ++d) c[d] = centre[d];
    std::vector<unsigned int> ids(k);
    std::vector<float> d2(k);
    check(fkd_search_knn(h_, c, 1, k, ids.data(), d2.data(), FKD_MEM_HOST));
    size_t m = 0;
    while (m < k && ids[m] != 0xffffffffu) ++m;
    ids.resize(m);
    d2.resize(m);
    if (dist2) *dist2 = d2;
    return ids;
  }

  std::vector<unsigned int> search_in_the_box(const Point& minPoint, const Point& maxPoint) override {
    return one(minPoint, maxPoint);
  }
  std::vector<unsigned int> search_in_the_box_BFS(const Point& minPoint, const Point& maxPoint) {
    return one(minPoint, maxPoint);
  }
  std::vector<unsigned int> search_in_the_box_branchless(const Point& minPoint, const Point& maxPoint) {
    return one(minPoint, maxPoint);
  }
  void search_in_the_box_recursive(const Point& minPoint, const Point& maxPoint,
                                   std::vector<unsigned int>& foundPoints, unsigned int = 0, int = 0) {
    std::vector<unsigned int> r = one(minPoint, maxPoint);
    foundPoints.insert(foundPoints.end(), r.begin(), r.end());
  }

  std::vector<unsigned int> search_in_the_box_multiple(const std::vector<Point>& minPoints,
                                                       const std::vector<Point>& maxPoints) override {
    std::vector<float> lo, hi;
    soa(minPoints, maxPoints, lo, hi);
    std::vector<unsigned int> counts(minPoints.size());
    check(fkd_search_count(h_, lo.data(), hi.data(), minPoints.size(), counts.data(), FKD_MEM_HOST));
    return counts;
  }

  // All boxes in one call: ids of box j are ids[offsets[j] .. offsets[j+1]).
  void search_in_the_box_batch(const std::vector<Point>& minPoints, const std::vector<Point>& maxPoints,
                               std::vector<uint64_t>& offsets, std::vector<unsigned int>& ids,
                               bool ordered = true) {
    std::vector<float> lo, hi;
    soa(minPoints, maxPoints, lo, hi);
    const uint64_t q = minPoints.size();
    std::vector<unsigned int> counts(q);
    check(fkd_search_count(h_, lo.data(), hi.data(), q, counts.data(), FKD_MEM_HOST));
    offsets.assign(q + 1, 0);
    for (uint64_t j = 0; j < q; ++j) offsets[j + 1] = offsets[j] + counts[j];
    ids.resize(offsets[q]);
    uint64_t total = 0;
    check(fkd_search(h_, lo.data(), hi.data(), q, offsets.data(), ids.data(), ids.size(), &total, ordered ? 1 : 0,
                     FKD_MEM_HOST));
  }

  std::vector<TYPE> const& getDimensionVector(const int dimension) override {
    sync_tables();
    if ((unsigned int)dimension < numberOfDimensions) return dims_[dimension];
    return dims_[0];  // FKDTree_cpu.h:210-211
  }
  std::vector<unsigned int> const& getIdVector() override {
    sync_tables();
    return tab_ids_;
  }

  fkd_tree handle() const { return h_; }

 private:
  static void check(fkd_status s) {
    if (s != FKD_OK) throw std::runtime_error(std::string("fkdtree_b200: ") + fkd_last_error());
  }

  static void soa(const std::vector<Point>& a, const std::vector<Point>& b, std::vector<float>& lo,
                  std::vector<float>& hi) {
    if (a.size() != b.size()) throw std::invalid_argument("minPoints and maxPoints differ in size");
    const size_t q = a.size();
    lo.resize(numberOfDimensions * q);
    hi.resize(numberOfDimensions * q);
    for (size_t j = 0; j < q; ++j)
      for (unsigned int c = 0; c < numberOfDimensions; ++c) {
        lo[c * q + j] = a[j][c];
        hi[c * q + j] = b[j][c];
      }
  }

  // One box, one library call: the result lands in a per-thread buffer sized
  // by the largest box this thread has seen; only a box larger than that
  // takes a second call (fkd_search reports the total with FKD_ERR_CAPACITY).
  std::vector<unsigned int> one(const Point& minPoint, const Point& maxPoint) {
    float lo[numberOfDimensions], hi[numberOfDimensions];
    for (unsigned int c = 0; c < numberOfDimensions; ++c) {
      lo[c] = minPoint[c];
      hi[c] = maxPoint[c];
    }
    thread_local std::vector<unsigned int> buf(256);
    uint64_t offsets[2] = {0, 0};
    uint64_t total = 0;
    fkd_status s = fkd_search(h_, lo, hi, 1, offsets, buf.data(), buf.size(), &total, 1, FKD_MEM_HOST);
    if (s == FKD_ERR_CAPACITY && total > buf.size()) {
      buf.resize(total + total / 2);
      s = fkd_search(h_, lo, hi, 1, offsets, buf.data(), buf.size(), &total, 1, FKD_MEM_HOST);
    }
    check(s);
    return std::vector<unsigned int>(buf.begin(), buf.begin() + total);
  }

  void sync_tables() {
    std::lock_guard<std::mutex> g(tables_mu_);
    if (synced_) return;
    std::vector<float> flat(numberOfDimensions * n_);
    tab_ids_.resize(n_);
    check(fkd_get_tables(h_, flat.data(), tab_ids_.data(), FKD_MEM_HOST));
    dims_.assign(numberOfDimensions, std::vector<TYPE>(n_));
    for (unsigned int c = 0; c < numberOfDimensions; ++c)
      for (size_t i = 0; i < n_; ++i) dims_[c][i] = flat[c * n_ + i];
    synced_ = true;
  }

  size_t n_;
  std::vector<Point> points_;
  fkd_tree h_ = nullptr;
  std::mutex tables_mu_;  // the lazy table download (getDimensionVector / getIdVector)
  bool synced_;
  std::vector<std::vector<TYPE>> dims_;
  std::vector<unsigned int> tab_ids_;
};

#endif  // FKDTREE_CUDA_H_
