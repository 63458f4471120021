/*
 * bvh.cpp - bounding-volume hierarchy over the candidate surfaces of a grain.
 *
 * The reference tests every surface of the current grain on every flight
 * (findCollisionSurface, src/RTMCphon.f90:1989-2096); a grain that holds a
 * triangulated mesh (tens of thousands of facets in the fill grain of a
 * bricks structure) makes that the whole cost.  Grains with many candidates
 * get a binned-SAH BVH here: top-down, 16 centroid bins per axis, surface
 * area cost, leaves of at most `leaf` surfaces (larger only at the depth
 * limit, which bounds the device traversal stack).
 *
 * Node layout (two float4 per node, 32 bytes, in the FP32 geometry blob):
 *   n0 = (lo.x, lo.y, lo.z, a)   n1 = (hi.x, hi.y, hi.z, b)
 *   internal: b = 0, children at node indices a and a + 1 (adjacent)
 *   leaf:     b = count > 0, surfaces cand[a .. a + b) of the blob's
 *             candidate list, which is reordered so every leaf is contiguous.
 * Boxes are padded by `pad` so the tolerant FP32 tests (t >= -eps, points
 * within eps of an edge) never hit a surface outside its node's box.
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ptg_internal.h"

namespace ptg {

namespace {

struct Box {
  float lo[3], hi[3];
  void reset() {
    for (int d = 0; d < 3; ++d) { lo[d] = 3.0e38f; hi[d] = -3.0e38f; }
  }
  void grow(const Box& b) {
    for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], b.lo[d]); hi[d] = std::max(hi[d], b.hi[d]); }
  }
  void grow(const float* p) {
    for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], p[d]); hi[d] = std::max(hi[d], p[d]); }
  }
  double area() const {
    const double x = std::max(0.0f, hi[0] - lo[0]), y = std::max(0.0f, hi[1] - lo[1]),
                 z = std::max(0.0f, hi[2] - lo[2]);
    return 2.0 * (x * y + y * z + z * x);
  }
};

struct Builder {
  const std::vector<Box>* prim;
  std::vector<float> cen;       /* 3 per primitive */
  std::vector<int> idx;         /* primitive order, permuted in place */
  std::vector<Box> nbox;
  std::vector<int> na, nb;      /* node words a, b (see layout) */
  int leaf, max_depth, base;    /* base: candidate index of idx[0] */

  int new_pair() {
    const int n = (int)nbox.size();
    nbox.resize(n + 2);
    na.resize(n + 2);
    nb.resize(n + 2);
    return n;
  }

  void make_leaf(int node, int begin, int end) {
    na[node] = base + begin;
    nb[node] = end - begin;
  }

  void build(int node, int begin, int end, int depth) {
    Box b, cb;
    b.reset();
    cb.reset();
    for (int i = begin; i < end; ++i) {
      b.grow((*prim)[idx[i]]);
      cb.grow(&cen[3 * idx[i]]);
    }
    nbox[node] = b;
    const int n = end - begin;
    if (n <= leaf || depth >= max_depth) { make_leaf(node, begin, end); return; }
    constexpr int kBins = 16;
    double best = 1e300;
    int bax = -1, bsplit = 0;
    for (int ax = 0; ax < 3; ++ax) {
      const float ext = cb.hi[ax] - cb.lo[ax];
      if (!(ext > 0.0f)) continue;
      Box bin[kBins];
      int cnt[kBins] = {0};
      for (auto& x : bin) x.reset();
      const float sc = kBins / ext;
      for (int i = begin; i < end; ++i) {
        int k = (int)((cen[3 * idx[i] + ax] - cb.lo[ax]) * sc);
        k = std::min(std::max(k, 0), kBins - 1);
        ++cnt[k];
        bin[k].grow((*prim)[idx[i]]);
      }
      double ra[kBins];
      int rc[kBins];
      Box acc;
      acc.reset();
      int c = 0;
      for (int k = kBins - 1; k > 0; --k) {
        acc.grow(bin[k]);
        c += cnt[k];
        ra[k] = acc.area();
        rc[k] = c;
      }
      acc.reset();
      c = 0;
      for (int k = 0; k < kBins - 1; ++k) {
        acc.grow(bin[k]);
        c += cnt[k];
        if (c == 0 || rc[k + 1] == 0) continue;
        const double cost = c * acc.area() + rc[k + 1] * ra[k + 1];
        if (cost < best) { best = cost; bax = ax; bsplit = k; }
      }
    }
    int mid;
    if (bax < 0) {
      /* coincident centroids: split by count */
      mid = begin + n / 2;
    } else {
      if (best >= n * b.area() && n <= 4 * leaf) { make_leaf(node, begin, end); return; }
      const float ext = cb.hi[bax] - cb.lo[bax];
      const float sc = kBins / ext;
      auto left = [&](int p) {
        int k = (int)((cen[3 * p + bax] - cb.lo[bax]) * sc);
        k = std::min(std::max(k, 0), kBins - 1);
        return k <= bsplit;
      };
      mid = (int)(std::partition(idx.begin() + begin, idx.begin() + end, left) - idx.begin());
      if (mid == begin || mid == end) mid = begin + n / 2;
    }
    const int c = new_pair();
    na[node] = c;
    nb[node] = 0;
    build(c, begin, mid, depth + 1);
    build(c + 1, mid, end, depth + 1);
  }
};

}  // namespace

int bvh_build(const std::vector<float>& lo, const std::vector<float>& hi, int leaf, int max_depth,
              int cand_base, int node_base, std::vector<float4>* nodes, std::vector<int>* order) {
  const int n = (int)(lo.size() / 3);
  std::vector<Box> prim(n);
  Builder B;
  B.prim = &prim;
  B.cen.resize(3 * (size_t)n);
  B.idx.resize(n);
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) {
      prim[i].lo[d] = lo[3 * i + d];
      prim[i].hi[d] = hi[3 * i + d];
      B.cen[3 * i + d] = 0.5f * (lo[3 * i + d] + hi[3 * i + d]);
    }
    B.idx[i] = i;
  }
  B.leaf = std::max(1, leaf);
  B.max_depth = max_depth;
  B.base = cand_base;
  B.new_pair();  /* root at 0; slot 1 unused so children pairs stay adjacent */
  B.build(0, 0, n, 0);
  const int nn = (int)B.nbox.size();
  nodes->resize(2 * (size_t)nn);
  for (int i = 0; i < nn; ++i) {
    float4 a = make_float4(B.nbox[i].lo[0], B.nbox[i].lo[1], B.nbox[i].lo[2], 0.0f);
    float4 b = make_float4(B.nbox[i].hi[0], B.nbox[i].hi[1], B.nbox[i].hi[2], 0.0f);
    const int aw = B.nb[i] > 0 ? B.na[i] : B.na[i] + node_base;
    memcpy(&a.w, &aw, 4);
    memcpy(&b.w, &B.nb[i], 4);
    (*nodes)[2 * i] = a;
    (*nodes)[2 * i + 1] = b;
  }
  *order = B.idx;
  return nn;
}

}  // namespace ptg
