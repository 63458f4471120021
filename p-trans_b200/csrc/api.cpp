/*
 * api.cpp - the C ABI of include/ptrans_gpu.h: device handles, task and
 * work-queue construction, kernel launches and the FP64 kappa assembly.
 *
 * The transport entry points replace the body of TransmissionFunction
 * (src/RTMCphon.f90:1544-1604); ptg_kappa additionally replaces effectiveMFP
 * (:2418-2451) and the kappa sum of fileoutput (:2645-2755).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "kernels.h"
#include "ptg_internal.h"

namespace {

/* Growable device buffer. */
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    if (ptg::alloc_should_fail()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

/* Pinned host staging for a call's tables: copied to the device
   asynchronously, reused once the copy recorded on `done` has finished. */
struct PinBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (ptg::alloc_should_fail()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

#define CU(x)                                                                \
  do {                                                                       \
    cudaError_t e_ = (x);                                                    \
    if (e_ != cudaSuccess) {                                                 \
      h->last_error = cudaGetErrorString(e_);                                \
      return e_ == cudaErrorMemoryAllocation ? PTG_ERR_NOMEM : PTG_ERR_CUDA; \
    }                                                                        \
  } while (0)

}  // namespace

struct ptg_handle {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  /* 0/1 around the transport, 2/3 around the reduction, 4 between the
     drain and tail kernels */
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  ptg_options opt;
  ptg::GeomSoA geom;
  ptg::SpecSoA spec;
  std::string last_error;
  ptg_stats last;
  /* FP64 geometry */
  std::vector<DevBuf*> owned;
  ptg::Geo64 g64;
  /* FP32 blob */
  DevBuf blob;
  ptg::GeoF32 g32;
  size_t blob_bytes = 0;
  /* work buffers */
  DevBuf task, chunk, counts, lost, stats, queue, order;
  /* pinned staging of the FP32 task table and queue order; h2d_done marks
     the end of their last copy */
  PinBuf pin_task, pin_order;
  cudaEvent_t h2d_done = nullptr;
  bool h2d_pending = false;
  /* FP32 tail phase: phonons the drain phase hands over */
  DevBuf tail;
  /* reduction */
  DevBuf red_coef, red_K, red_W, red_mfp, red_bin, red_grid, red_tc, red_kv, red_bw, red_bv,
      red_emfp, red_trans, red_result;
  /* adjoint: list of transmitted samples, per-sample weights, accumulators */
  DevBuf adj_list, adj_w, adj_acc;
  /* trace replay: position offsets, counts, exit sides, positions */
  DevBuf tr_off, tr_npos, tr_end, tr_pos;
  unsigned long long list_n = 0, mismatch = 0;
  bool fp32_split = false;  /* the last transport was the FP32 drain (+ tail) */
  int tail_cap = 0;          /* its tail-list capacity (0: no tail phase)       */
  ~ptg_handle() {
    for (DevBuf* b : owned) { b->release(); delete b; }
    DevBuf* all[] = {&blob, &task, &chunk, &counts, &lost, &stats, &queue, &red_coef, &red_K,
                     &red_W, &red_mfp, &red_bin, &red_grid, &red_tc, &red_kv, &red_bw, &red_bv,
                     &red_emfp, &red_trans, &red_result, &adj_list, &adj_w, &adj_acc,
                     &tr_off, &tr_npos, &tr_end, &tr_pos, &tail, &order};
    for (DevBuf* b : all) b->release();
    if (stream) cudaStreamSynchronize(stream);
    pin_task.release();
    pin_order.release();
    for (cudaEvent_t e : ev) if (e) cudaEventDestroy(e);
    if (h2d_done) cudaEventDestroy(h2d_done);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class T>
int upload(ptg_handle* h, const std::vector<T>& v, const T** out) {
  DevBuf* b = new DevBuf();
  h->owned.push_back(b);
  const size_t bytes = sizeof(T) * (v.size() ? v.size() : 1);
  CU(b->ensure(bytes));
  if (!v.empty()) CU(cudaMemcpy(b->p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  *out = static_cast<const T*>(b->p);
  return PTG_OK;
}

/* ---- FP32 geometry blob -------------------------------------------------- */

inline float4 f4(double a, double b, double c, double d) {
  return make_float4((float)a, (float)b, (float)c, (float)d);
}
inline float4 i4(int a, int b, int c, int d) {
  float4 v;
  memcpy(&v.x, &a, 4);
  memcpy(&v.y, &b, 4);
  memcpy(&v.z, &c, 4);
  memcpy(&v.w, &d, 4);
  return v;
}

}  // namespace

namespace ptg {

/* The FP32 geometry blob of a built geometry (host copy) and its layout. */
int blob_from_geometry(const GeomSoA& G, int bvh_leaf, std::vector<float4>* out,
                       BlobLayout* lay_out, std::string* why) {
  const int ns = G.nsurf(), ngt = G.ngrain_total();
  std::vector<float4> hot(2 * (size_t)ns), cold(3 * (size_t)ns), edges;
  std::vector<int> geom_id(ns);
  for (int s = 0; s < ns; ++s) geom_id[s] = s;
  /* a fill-grain quadric is the same physical surface as its brick's */
  if (G.kind_grain == PTG_GRAIN_BRICKS && G.igrain_fill > 0) {
    const int fb = G.grain_begin[G.igrain_fill], fe = G.grain_begin[G.igrain_fill + 1];
    for (int s = fb; s < fe; ++s) {
      if (G.shape[s] == PTG_SHAPE_POLYGON) continue;
      for (int t = G.grain_begin[1]; t < fb; ++t) {
        bool same_axis = true;
        if (G.shape[s] == PTG_SHAPE_CAPPED && G.shape[t] == PTG_SHAPE_CAPPED) {
          const double* vs = &G.vertex[3 * (size_t)G.vertex_begin[s]];
          const double* vt = &G.vertex[3 * (size_t)G.vertex_begin[t]];
          for (int d = 0; d < 6; ++d) same_axis = same_axis && vs[d] == vt[d];
        }
        if (G.shape[t] == G.shape[s] && G.radius[t] == G.radius[s] && same_axis &&
            G.center[3 * t] == G.center[3 * s] && G.center[3 * t + 1] == G.center[3 * s + 1] &&
            G.center[3 * t + 2] == G.center[3 * s + 2]) {
          geom_id[s] = t;
          break;
        }
      }
    }
  }
  for (int g = 0; g < ngt; ++g) {
    for (int s = G.grain_begin[g]; s < G.grain_begin[g + 1]; ++s) {
      const double* n = &G.normal[3 * s];
      const double* t = &G.tangent[9 * s];
      const int meta = (G.kind_trans[s] & 0xff) | (G.grain_outside[s] << 8);
      cold[3 * s + 0] = f4(t[0], t[1], t[2], G.specularity[s]);
      cold[3 * s + 1] = f4(t[3], t[4], t[5], G.trans_param[s]);
      cold[3 * s + 2] = f4(n[0], n[1], n[2], 0.0);
      memcpy(&cold[3 * s + 2].w, &meta, 4);
      const double* c = &G.center[3 * s];
      if (G.shape[s] == PTG_SHAPE_POLYGON) {
        const int nv = G.nvertex[s];
        const double* v = &G.vertex[3 * (size_t)G.vertex_begin[s]];
        /* winding normal: sum of the consecutive-triple cross products */
        double wn[3] = {0, 0, 0};
        for (int i = 0; i < nv; ++i) {
          const double* p0 = v + 3 * i;
          const double* p1 = v + 3 * ((i + 1) % nv);
          const double* p2 = v + 3 * ((i + 2) % nv);
          double a[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
          double b[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
          wn[0] += a[1] * b[2] - a[2] * b[1];
          wn[1] += a[2] * b[0] - a[0] * b[2];
          wn[2] += a[0] * b[1] - a[1] * b[0];
        }
        double ln = sqrt(wn[0] * wn[0] + wn[1] * wn[1] + wn[2] * wn[2]);
        if (!(ln > 0.0)) { *why = "degenerate polygon"; return PTG_ERR_INVALID; }
        for (int d = 0; d < 3; ++d) wn[d] /= ln;
        const int e0 = (int)edges.size();
        for (int i = 0; i < nv; ++i) {
          const double* p0 = v + 3 * i;
          const double* p1 = v + 3 * (i + 1);
          double e[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
          double m[3] = {wn[1] * e[2] - wn[2] * e[1], wn[2] * e[0] - wn[0] * e[2],
                         wn[0] * e[1] - wn[1] * e[0]};
          double lm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
          if (!(lm > 0.0)) { lm = 1.0; }
          for (int d = 0; d < 3; ++d) m[d] /= lm;
          edges.push_back(f4(m[0], m[1], m[2], m[0] * p0[0] + m[1] * p0[1] + m[2] * p0[2]));
        }
        const double d0 = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
        hot[2 * s] = f4(n[0], n[1], n[2], d0);
        hot[2 * s + 1] = i4(ptg::REC_POLY, e0, nv, geom_id[s]);
      } else if (G.shape[s] == PTG_SHAPE_SPHERE) {
        const int interior = (g != G.igrain_fill) ? ptg::REC_INTERIOR : 0;
        hot[2 * s] = f4(c[0], c[1], c[2], G.radius[s]);
        hot[2 * s + 1] = i4(ptg::REC_SPHERE | interior, 0, 0, geom_id[s]);
      } else if (G.shape[s] == PTG_SHAPE_CAPPED) {
        const int interior = (g != G.igrain_fill) ? ptg::REC_INTERIOR : 0;
        const double* v = &G.vertex[3 * (size_t)G.vertex_begin[s]];
        double e[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
        const double len = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        const int e0 = (int)edges.size();
        edges.push_back(f4(e[0] / len, e[1] / len, e[2] / len, 0.5 * len));
        hot[2 * s] = f4(c[0], c[1], c[2], G.radius[s]);
        hot[2 * s + 1] = i4(ptg::REC_CAP | interior, e0, 0, geom_id[s]);
      } else {
        const int interior = (g != G.igrain_fill) ? ptg::REC_INTERIOR : 0;
        hot[2 * s] = f4(c[0], c[1], G.radius[s], 0.0);
        hot[2 * s + 1] = i4(ptg::REC_CYL | interior, 0, 0, geom_id[s]);
      }
    }
  }
  std::vector<int> cb(ngt + 1, 0), cand;
  for (int g = 0; g < ngt; ++g) {
    cb[g] = (int)cand.size();
    if (g == 0) continue;
    for (int s = G.grain_begin[g]; s < G.grain_begin[g + 1]; ++s)
      if (G.internal[s]) cand.push_back(s);
  }
  cb[ngt] = (int)cand.size();
  /* BVH over the candidates of every large grain; its leaves reorder the
     grain's candidate list */
  std::vector<int> root(ngt, -1);
  std::vector<float4> nodes;
  if (bvh_leaf >= 0) {
    const int leaf = bvh_leaf > 0 ? bvh_leaf : kBvhDefaultLeaf;
    const double S = std::max(G.box[0], std::max(G.box[1], G.box[2]));
    const double pad = 4.0 * S / 1048576.0;  /* 4 eps of the FP32 tests */
    for (int g = 1; g < ngt; ++g) {
      const int n = cb[g + 1] - cb[g];
      if (n <= kBvhMinCand) continue;
      std::vector<float> lo(3 * (size_t)n), hi(3 * (size_t)n);
      for (int i = 0; i < n; ++i) {
        const int s = cand[cb[g] + i];
        double l[3], h[3];
        if (G.shape[s] == PTG_SHAPE_POLYGON) {
          for (int d = 0; d < 3; ++d) { l[d] = 1e300; h[d] = -1e300; }
          const double* v = &G.vertex[3 * (size_t)G.vertex_begin[s]];
          for (int k = 0; k < G.nvertex[s]; ++k)
            for (int d = 0; d < 3; ++d) {
              l[d] = std::min(l[d], v[3 * k + d]);
              h[d] = std::max(h[d], v[3 * k + d]);
            }
        } else if (G.shape[s] == PTG_SHAPE_CAPPED) {
          /* extent per axis: half length times |a_d| + radius times sin */
          const double* c = &G.center[3 * s];
          const double* v = &G.vertex[3 * (size_t)G.vertex_begin[s]];
          double e[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
          const double len = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
          for (int d = 0; d < 3; ++d) {
            const double ad = fabs(e[d]) / len;
            const double ext = 0.5 * len * ad + G.radius[s] * sqrt(std::max(0.0, 1.0 - ad * ad));
            l[d] = c[d] - ext;
            h[d] = c[d] + ext;
          }
        } else {
          const double* c = &G.center[3 * s];
          const double r = G.radius[s];
          for (int d = 0; d < 3; ++d) { l[d] = c[d] - r; h[d] = c[d] + r; }
          if (G.shape[s] == PTG_SHAPE_CYLINDER) { l[2] = 0.0; h[2] = G.box[2]; }
        }
        for (int d = 0; d < 3; ++d) {
          /* rounded outwards after the pad */
          lo[3 * i + d] = std::nextafter((float)(l[d] - pad), -3.0e38f);
          hi[3 * i + d] = std::nextafter((float)(h[d] + pad), 3.0e38f);
        }
      }
      std::vector<float4> gn;
      std::vector<int> order;
      const int node_base = (int)(nodes.size() / 2);
      bvh_build(lo, hi, leaf, 30, cb[g], node_base, &gn, &order);
      std::vector<int> seg(cand.begin() + cb[g], cand.begin() + cb[g + 1]);
      for (int i = 0; i < n; ++i) cand[cb[g] + i] = seg[order[i]];
      root[g] = node_base;
      nodes.insert(nodes.end(), gn.begin(), gn.end());
    }
  }
  if (!nodes.empty()) {
    /* breadth first over all grains' trees (every root first, then level
       by level): the front of the node region holds the top levels of
       every tree, the part staged in shared memory when the whole blob is
       too large to stage.  Child pairs stay adjacent; a root keeps an
       unused partner slot. */
    const int nn = (int)(nodes.size() / 2);
    auto word = [](const float4& v) { int w; memcpy(&w, &v.w, 4); return w; };
    std::vector<int> newidx(nn, -1), queue;
    queue.reserve(nn);
    int next = 0;
    for (int g = 1; g < ngt; ++g)
      if (root[g] >= 0) {
        newidx[root[g]] = next;
        next += 2;
        queue.push_back(root[g]);
      }
    for (size_t qi = 0; qi < queue.size(); ++qi) {
      const int o = queue[qi];
      if (word(nodes[2 * (size_t)o + 1]) != 0) continue;  /* leaf */
      const int a = word(nodes[2 * (size_t)o]);
      newidx[a] = next;
      newidx[a + 1] = next + 1;
      next += 2;
      queue.push_back(a);
      queue.push_back(a + 1);
    }
    std::vector<float4> bfs(2 * (size_t)next, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    for (int o = 0; o < nn; ++o) {
      if (newidx[o] < 0) continue;
      float4 a = nodes[2 * (size_t)o];
      const float4 b = nodes[2 * (size_t)o + 1];
      if (word(b) == 0) {
        const int na = newidx[word(a)];
        memcpy(&a.w, &na, 4);
      }
      bfs[2 * (size_t)newidx[o]] = a;
      bfs[2 * (size_t)newidx[o] + 1] = b;
    }
    for (int g = 1; g < ngt; ++g)
      if (root[g] >= 0) root[g] = newidx[root[g]];
    nodes.swap(bfs);
  }
  std::vector<float4> start;
  for (int g = 1; g <= G.ngrain; ++g) {
    if (!G.grain_incident[g]) continue;
    if (G.kind_grain == PTG_GRAIN_VORONOI) {
      float4 v = f4(G.grain_generatrix[3 * g], G.grain_generatrix[3 * g + 1],
                    G.grain_generatrix[3 * g + 2], 0.0);
      memcpy(&v.w, &g, 4);
      start.push_back(v);
    } else {
      for (int s = G.grain_begin[g]; s < G.grain_begin[g + 1]; ++s)
        if (G.incident[s] && G.shape[s] == PTG_SHAPE_POLYGON) start.push_back(i4(s, g, 0, 0));
    }
  }
  auto units_of_ints = [](size_t n) { return (int)((n * 4 + 15) / 16); };
  ptg::BlobLayout L;
  L.hot = 0;
  L.cold = L.hot + 2 * ns;
  L.edge = L.cold + 3 * ns;
  L.cand_begin = L.edge + (int)edges.size();
  L.cand = L.cand_begin + units_of_ints(cb.size());
  L.start = L.cand + units_of_ints(cand.size() ? cand.size() : 1);
  L.bvh_root = L.start + (int)(start.size() ? start.size() : 1);
  L.bvh_node = L.bvh_root + units_of_ints(root.size());
  L.total = L.bvh_node + (int)(nodes.size() ? nodes.size() : 1);
  L.nbvh = (int)(nodes.size() / 2);
  L.ncap = 0;
  for (int s = 0; s < ns; ++s) L.ncap += G.shape[s] == PTG_SHAPE_CAPPED ? 1 : 0;
  L.nstart = (int)start.size();
  std::vector<float4> blob((size_t)L.total, make_float4(0, 0, 0, 0));
  std::copy(hot.begin(), hot.end(), blob.begin() + L.hot);
  std::copy(cold.begin(), cold.end(), blob.begin() + L.cold);
  std::copy(edges.begin(), edges.end(), blob.begin() + L.edge);
  memcpy(&blob[L.cand_begin], cb.data(), cb.size() * 4);
  if (!cand.empty()) memcpy(&blob[L.cand], cand.data(), cand.size() * 4);
  std::copy(start.begin(), start.end(), blob.begin() + L.start);
  memcpy(&blob[L.bvh_root], root.data(), root.size() * 4);
  std::copy(nodes.begin(), nodes.end(), blob.begin() + L.bvh_node);
  *out = std::move(blob);
  *lay_out = L;
  return PTG_OK;
}

bool handle_has_bvh(const ptg_handle* h) {
  const GeomSoA& G = h->geom;
  for (int g = 1; g < G.ngrain_total(); ++g) {
    int n = 0;
    for (int s = G.grain_begin[g]; s < G.grain_begin[g + 1]; ++s) n += G.internal[s] ? 1 : 0;
    if (n > kBvhMinCand) return true;
  }
  return false;
}

}  // namespace ptg

namespace {

int build_blob(ptg_handle* h) {
  const ptg::GeomSoA& G = h->geom;
  std::vector<float4> blob;
  ptg::BlobLayout L;
  std::string why;
  int st = ptg::blob_from_geometry(G, h->opt.bvh_leaf, &blob, &L, &why);
  if (st != PTG_OK) { h->last_error = why; return st; }
  h->blob_bytes = blob.size() * 16;
  CU(h->blob.ensure(h->blob_bytes));
  CU(cudaMemcpy(h->blob.p, blob.data(), h->blob_bytes, cudaMemcpyHostToDevice));
  ptg::GeoF32& g32 = h->g32;
  g32.blob = h->blob.as<const float4>();
  g32.lay = L;
  for (int d = 0; d < 3; ++d) g32.box[d] = (float)G.box[d];
  g32.scope[0] = (float)G.scope[0];
  g32.scope[1] = (float)G.scope[1];
  const double S = std::max(G.box[0], std::max(G.box[1], G.box[2]));
  g32.eps = (float)(S * (1.0 / 1048576.0));
  g32.periodic_mask = 0;
  for (int f = 0; f < 6; ++f)
    if (G.face_kind[f] == PTG_FACE_PERIODIC) g32.periodic_mask |= 1 << f;
  g32.kind_grain = G.kind_grain;
  g32.igrain_fill = G.igrain_fill;
  g32.nmaterial = G.nmaterial;
  g32.stage_smem = h->blob_bytes <= 96 * 1024 ? 1 : 0;
  g32.has_ext = (L.nbvh > 0 || L.ncap > 0) ? 1 : 0;
  /* a blob too large to stage keeps the top levels of its BVHs (the front of
     the breadth-first node region) in shared memory */
  g32.node_stage = (!g32.stage_smem && L.nbvh > 0) ? std::min(2 * L.nbvh, ptg::kNodeStageUnits) : 0;
  return PTG_OK;
}

int build_geo64(ptg_handle* h) {
  const ptg::GeomSoA& G = h->geom;
  ptg::Geo64& g = h->g64;
  int st;
  if ((st = upload(h, G.vertex, &g.vertex))) return st;
  if ((st = upload(h, G.normal, &g.normal))) return st;
  if ((st = upload(h, G.tangent, &g.tangent))) return st;
  if ((st = upload(h, G.center, &g.center))) return st;
  if ((st = upload(h, G.radius, &g.radius))) return st;
  if ((st = upload(h, G.specularity, &g.spec))) return st;
  if ((st = upload(h, G.trans_param, &g.tparam))) return st;
  if ((st = upload(h, G.shape, &g.shape))) return st;
  if ((st = upload(h, G.nvertex, &g.nvertex))) return st;
  if ((st = upload(h, G.vertex_begin, &g.vbegin))) return st;
  if ((st = upload(h, G.kind_trans, &g.kind_trans))) return st;
  if ((st = upload(h, G.grain_outside, &g.gout))) return st;
  if ((st = upload(h, G.internal, &g.internal))) return st;
  if ((st = upload(h, G.incident, &g.incident))) return st;
  if ((st = upload(h, G.grain_begin, &g.grain_begin))) return st;
  if ((st = upload(h, G.grain_incident, &g.grain_incident))) return st;
  if ((st = upload(h, G.grain_generatrix, &g.grain_gen))) return st;
  for (int d = 0; d < 3; ++d) g.box[d] = G.box[d];
  g.scope[0] = G.scope[0];
  g.scope[1] = G.scope[1];
  for (int f = 0; f < 6; ++f) g.face_kind[f] = G.face_kind[f];
  g.kind_grain = G.kind_grain;
  g.ngrain = G.ngrain;
  g.igrain_fill = G.igrain_fill;
  g.nmaterial = G.nmaterial;
  g.max_omega = h->spec.max_omega;
  return PTG_OK;
}

/* ---- one transport pass over a task list --------------------------------- */

struct Transport {
  int64_t ntask = 0;
  int64_t np = 0, np_local = 0;
  int32_t rank = 0, nranks = 1;
  uint64_t seed = 0;
  int32_t stream = 0;
  int32_t precision = PTG_PREC_FP32;
  const std::vector<ptg::TaskHost>* tasks = nullptr;
  /* tasks whose MFP can differ: task t has the MFP of task t % npair (the
     (mode, grid point) pairs of the first angle; 0: every task) */
  int64_t npair = 0;
  /* persistent kernel mode and the adjoint buffers */
  int mode = ptg::MODE_FORWARD;
  unsigned long long* tlist = nullptr;
  unsigned long long tlist_cap = 0;
  const unsigned long long* alist = nullptr;
  long long alist_n = 0;
  const float* wsample = nullptr;
  double* adj = nullptr;
  /* trace replay (mode 3) */
  float* trace = nullptr;
  const long long* trace_off = nullptr;
  long long* trace_npos = nullptr;
  int* trace_end = nullptr;
};

int run_transport(ptg_handle* h, const Transport& T) {
  ptg::NvtxRange nvtx(T.mode == ptg::MODE_LIST      ? "ptg transport: list"
                      : T.mode == ptg::MODE_ADJOINT ? "ptg transport: adjoint replay"
                      : T.mode == ptg::MODE_TRACE   ? "ptg transport: trace replay"
                                                    : "ptg transport");
  const int64_t ntask = T.ntask;
  CU(cudaSetDevice(h->device));
  CU(h->counts.ensure(sizeof(unsigned long long) * ntask));
  CU(h->lost.ensure(sizeof(unsigned long long) * ntask));
  CU(h->stats.ensure(sizeof(unsigned long long) * ptg::kStatSlots));
  CU(h->queue.ensure(sizeof(int) * 8));
  CU(cudaMemsetAsync(h->counts.p, 0, sizeof(unsigned long long) * ntask, h->stream));
  CU(cudaMemsetAsync(h->lost.p, 0, sizeof(unsigned long long) * ntask, h->stream));
  CU(cudaMemsetAsync(h->stats.p, 0, sizeof(unsigned long long) * ptg::kStatSlots, h->stream));
  /* stats[5], stats[6] collect minima of the global timer */
  CU(cudaMemsetAsync(h->stats.as<unsigned long long>() + 5, 0xFF, sizeof(unsigned long long) * 2,
                     h->stream));
  CU(cudaMemsetAsync(h->queue.p, 0, sizeof(int) * 8, h->stream));
  const int64_t maxf = h->opt.max_flights > 0 ? h->opt.max_flights : 10000000LL;
  memset(&h->last, 0, sizeof(h->last));
  if (T.precision == PTG_PREC_FP64) {
    std::vector<ptg::Task64> t64(ntask);
    for (int64_t i = 0; i < ntask; ++i) {
      const ptg::TaskHost& th = (*T.tasks)[i];
      t64[i] = {th.lambda, th.cth, th.sth, th.omega};
    }
    CU(h->task.ensure(sizeof(ptg::Task64) * ntask));
    CU(cudaMemcpyAsync(h->task.p, t64.data(), sizeof(ptg::Task64) * ntask, cudaMemcpyHostToDevice,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));  /* t64 is a local buffer */
    h->last.h2d_bytes += sizeof(ptg::Task64) * ntask;
    ptg::Run64 r;
    memset(&r, 0, sizeof(r));
    r.task = h->task.as<const ptg::Task64>();
    r.ntask = ntask;
    r.np = T.np;
    r.np_local = T.np_local;
    r.rank = T.rank;
    r.nranks = T.nranks;
    r.k0 = (uint32_t)T.seed;
    r.k1 = (uint32_t)(T.seed >> 32);
    r.c1 = ((uint32_t)T.stream) << 8;
    r.max_flights = maxf;
    r.ref_quirks = h->opt.ref_quirks;
    r.counts = h->counts.as<unsigned long long>();
    r.lost = h->lost.as<unsigned long long>();
    r.stats = h->stats.as<unsigned long long>();
    r.replay_task = -1;
    CU(cudaEventRecord(h->ev[0], h->stream));
    int grid = 0, block = 0;
    CU(ptg::launch_plain_fp64(h->g64, r, h->stream, &grid, &block));
    CU(cudaEventRecord(h->ev[1], h->stream));
    h->last.grid = grid;
    h->last.block = block;
    h->last.launches = 1;
    h->fp32_split = false;
  } else {
    /* the FP32 task table and the queue order (longest expected
       trajectories first: ascending MFP) are written to pinned staging and
       copied without a host wait; the chunk table (task, first local
       particle, count) is expanded from the order on the device.  The MFP
       depends on (mode, grid point) only, so those pairs are sorted and
       every angle's task follows its pair; equal MFPs keep index order. */
    if (h->h2d_pending) {
      CU(cudaEventSynchronize(h->h2d_done));
      h->h2d_pending = false;
    }
    CU(h->pin_task.ensure(sizeof(float4) * (ntask > 0 ? ntask : 1)));
    CU(h->pin_order.ensure(sizeof(int) * (ntask > 0 ? ntask : 1)));
    float4* t32 = h->pin_task.as<float4>();
    int* order = h->pin_order.as<int>();
    const int64_t npair = T.npair > 0 ? std::min<int64_t>(ntask, T.npair) : ntask;
    std::vector<int64_t> pairs;
    pairs.reserve(npair);
    for (int64_t i = 0; i < ntask; ++i) {
      const ptg::TaskHost& th = (*T.tasks)[i];
      float lam = th.lambda == 1.0e10 ? INFINITY : (float)th.lambda;
      if (!(th.lambda > 0.0)) lam = 0.0f;
      t32[i] = make_float4(lam, (float)th.cth, (float)th.sth,
                           (float)(th.omega / h->spec.max_omega));
      if (i < npair && th.lambda > 0.0) pairs.push_back(i);
    }
    std::stable_sort(pairs.begin(), pairs.end(), [&](int64_t a, int64_t b) {
      return (*T.tasks)[a].lambda < (*T.tasks)[b].lambda;
    });
    int64_t norder = 0;
    const int64_t nrep = npair > 0 ? (ntask + npair - 1) / npair : 0;
    for (int64_t pi : pairs)
      for (int64_t k = 0; k < nrep; ++k) {
        const int64_t t = pi + k * npair;
        if (t < ntask) order[norder++] = (int)t;
      }
    const int64_t csz = h->opt.chunk > 0 ? h->opt.chunk : 64;
    const int64_t per_task = T.np_local > 0 ? (T.np_local + csz - 1) / csz : 0;
    const int64_t nchunk = norder * per_task;
    if (nchunk > 2147483647LL) { h->last_error = "too many chunks"; return PTG_ERR_INVALID; }
    CU(h->task.ensure(sizeof(float4) * ntask));
    CU(h->order.ensure(sizeof(int) * (norder > 0 ? norder : 1)));
    CU(h->chunk.ensure(sizeof(int4) * (nchunk + 1)));
    CU(cudaMemcpyAsync(h->task.p, t32, sizeof(float4) * ntask, cudaMemcpyHostToDevice, h->stream));
    if (norder > 0)
      CU(cudaMemcpyAsync(h->order.p, order, sizeof(int) * norder, cudaMemcpyHostToDevice, h->stream));
    CU(cudaEventRecord(h->h2d_done, h->stream));
    h->h2d_pending = true;
    /* the timed transport starts here, with the tables resident: the chunk
       expansion is part of it */
    CU(cudaEventRecord(h->ev[0], h->stream));
    if (nchunk > 0)
      CU(ptg::launch_expand_chunks(h->order.as<const int>(), (int)norder, (int)per_task, (int)csz,
                                   (int)T.np_local, h->chunk.as<int4>(), h->stream));
    h->last.h2d_bytes += sizeof(float4) * ntask + sizeof(int) * norder;
    ptg::RunF32 r;
    memset(&r, 0, sizeof(r));
    r.task = h->task.as<const float4>();
    r.chunk = h->chunk.as<const int4>();
    r.nchunk = (int32_t)nchunk;
    r.np = T.np;
    r.rank = T.rank;
    r.nranks = T.nranks;
    r.k0 = (uint32_t)T.seed;
    r.k1 = (uint32_t)(T.seed >> 32);
    r.c1 = ((uint32_t)T.stream) << 8;
    r.max_flights = (uint32_t)std::min<int64_t>(maxf, 4294967295LL);
    r.ref_quirks = h->opt.ref_quirks;
    /* defaults: refill once 2 lanes are idle; at most 8 fast-path flights
       per lane and iteration (a lane that loops longer holds its warp's
       other lanes: 16 fast steps cost 13.6 ms of drain on the thin film
       against 11.1 ms for 8) */
    int rt = h->opt.regen_threshold > 0 ? h->opt.regen_threshold : ptg::kDefaultRegen;
    r.regen_threshold = rt > 32 ? 32 : rt;
    r.fast_steps = (h->opt.tune_flags & 1) ? 0 : (h->opt.fast_steps > 0 ? h->opt.fast_steps : ptg::default_fast_steps(h->g32));
    const double lmin = std::min(h->geom.box[0], std::min(h->geom.box[1], h->geom.box[2]));
    r.fast_lambda_max = (float)(0.1 * lmin);
    /* tune_flags bit 1 turns the tail phase off; 0 selects 32 lanes (every
       diffusive phonon still alive when a warp finds the queue dry) */
    r.coop_lanes = (h->opt.tune_flags & 2) ? 0 : (h->opt.coop_lanes > 0 ? std::min(h->opt.coop_lanes, 32) : 32);
    r.stage_test = (h->opt.tune_flags & 4) ? 1 : 0;
    r.counts = h->counts.as<unsigned long long>();
    r.lost = h->lost.as<unsigned long long>();
    r.stats = h->stats.as<unsigned long long>();
    r.queue = h->queue.as<int>();
    r.tlist = T.tlist;
    r.tlist_cap = T.tlist_cap;
    r.alist = T.alist;
    r.alist_n = T.alist_n;
    r.wsample = T.wsample;
    r.adj = T.adj;
    r.trace = T.trace;
    r.trace_off = T.trace_off;
    r.trace_npos = T.trace_npos;
    r.trace_end = T.trace_end;
    r.nsurf = h->geom.nsurf();
    const int bs = h->opt.block_size;
    const int block = (bs >= 32 && bs <= 256 && bs % 32 == 0) ? bs : 256;
    const size_t smem = ptg::dynamic_smem_bytes(h->g32, h->blob_bytes);
    int bps = 0;
    CU(ptg::persistent_occupancy(block, smem, &bps, T.mode, h->g32.has_ext != 0, h->g32.stage_smem != 0));
    if (h->opt.blocks_per_sm > 0 && h->opt.blocks_per_sm < bps) bps = h->opt.blocks_per_sm;
    if (bps < 1) bps = 1;
    const int grid = h->num_sms * bps;
    /* a lane hands over at most one phonon (no refill once the queue is
       dry), so the drain grid's lanes bound the tail list */
    const bool tail = r.coop_lanes > 0 && T.mode != ptg::MODE_TRACE;
    if (tail) {
      /* the list, then the order the tail phase takes it in */
      CU(h->tail.ensure((sizeof(float4) * ptg::kTailUnits + sizeof(int)) * (size_t)grid * block +
                        sizeof(int) * ptg::kTailOrderExtra));
      r.tail = h->tail.as<float4>();
      r.tail_cap = grid * block;
      r.tail_order = reinterpret_cast<int*>(r.tail + (size_t)ptg::kTailUnits * r.tail_cap);
    }
    int tgrid = 0;
    if (tail) {
      int tbps = 0;
      CU(ptg::tail_occupancy(block, smem, &tbps, T.mode, h->g32.has_ext != 0, h->g32.stage_smem != 0));
      tgrid = h->num_sms * (tbps < 1 ? 1 : tbps);
    }
    const bool work = (T.mode == ptg::MODE_ADJOINT || T.mode == ptg::MODE_TRACE) ? T.alist_n > 0
                                                                                   : r.nchunk > 0;
    if (work) {
      CU(ptg::launch_persistent_fp32(h->g32, r, grid, block, smem, h->stream, T.mode));
      CU(cudaEventRecord(h->ev[4], h->stream));
      if (tail) {
        CU(ptg::launch_tail_order(r, h->g32.box[0], h->stream));
        CU(ptg::launch_tail_fp32(h->g32, r, tgrid, block, smem, h->stream, T.mode));
      }
    }
    CU(cudaEventRecord(h->ev[1], h->stream));
    h->last.grid = grid;
    h->last.block = block;
    h->last.launches = (work ? (tail ? 4 : 1) : 0) + (r.nchunk > 0 ? 1 : 0);
    h->fp32_split = work;
    h->tail_cap = tail ? r.tail_cap : 0;
  }
  return PTG_OK;
}

int finish_stats(ptg_handle* h) {
  unsigned long long st[ptg::kStatSlots];
  int qerr[8];
  CU(cudaMemcpyAsync(st, h->stats.p, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaMemcpyAsync(qerr, h->queue.p, sizeof(qerr), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  float ms = 0.f;
  CU(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
  h->last.d2h_bytes += sizeof(st) + sizeof(qerr);
  h->last.flights = st[0];
  h->last.lost = st[1];
  h->last.capped = st[2];
  h->last.samples = st[3];
  h->last.kernel_ms = ms;
  h->last.max_traj_flights = st[4];
  h->last.full_flights = st[8];
  h->last.safe_balls = st[9];
  h->last.coop_rounds = st[12];
  h->last.coop_flights = st[13];
  h->last.box_tests = st[14];
  h->last.surface_tests = st[15];
  h->last.drain_kernel_ms = h->last.tail_kernel_ms = 0.0;
  h->last.tail_phonons = h->last.tail_flights = h->last.tail_refused = 0;
  if (h->fp32_split) {
    float dms = 0.f;
    CU(cudaEventElapsedTime(&dms, h->ev[0], h->ev[4]));
    h->last.drain_kernel_ms = dms;
    h->last.tail_kernel_ms = ms - dms;
    ptg::tail_counts(qerr, h->tail_cap, &h->last.tail_phonons, &h->last.tail_refused);
    h->last.tail_flights = st[17] >= st[16] ? st[17] - st[16] : 0;
  }
  h->list_n = st[10];
  h->mismatch = st[11];
  if (st[5] != ~0ull && st[7] >= st[5]) {
    const unsigned long long drain = st[6] != ~0ull ? st[6] : st[7];
    h->last.drain_ms = (double)(drain - st[5]) * 1e-6;
    h->last.tail_ms = (double)(st[7] - drain) * 1e-6;
  }
  if (qerr[1] != 0) { h->last_error = "shared-memory staging wait timed out"; return PTG_ERR_TIMEOUT; }
  return PTG_OK;
}

int64_t np_local_of(int64_t np, int32_t rank, int32_t nranks) {
  return np > rank ? (np - rank + nranks - 1) / nranks : 0;
}

int check_lost(ptg_handle* h) {
  if (h->opt.lost_limit > 0.0 && h->last.samples > 0 &&
      (double)h->last.lost > h->opt.lost_limit * (double)h->last.samples) {
    h->last_error = "lost-phonon fraction above the limit";
    return PTG_ERR_LOST;
  }
  return PTG_OK;
}

}  // namespace

namespace ptg {

/* effectiveMFP + the kappa sum of fileoutput from transmitted counts (host
   FP64), with the binomial standard errors and per-bin transmission; wtask
   (optional) receives d kappa / d T_task for every task and dk_ds_an the
   analytic part of d kappa / d s (the bulk-MFP dependence of the
   Matthiessen and grid-interpolation rules). */
int assemble_host(const ptg::SpecSoA& S, const ptg_run* run, double box_x, const uint64_t* counts,
                  ptg_kappa_out* out, std::vector<double>* wtask, double* dk_ds_an) {
  const int ns = run->kind_mfp == PTG_MFP_GRID ? run->nmfp : 1;
  const int na = run->nangle;
  const int64_t nm = S.nmode();
  ptg::ModeConst mc;
  ptg::mode_constants(S, run, &mc);
  std::vector<double> coef;
  double dS = 0.0;
  ptg::simpson_weights(na, box_x, &coef, &dS);
  const double tnorm = 0.75 * box_x;
  const double np = (double)run->np;
  double kappa = 0.0, kvar = 0.0, dks = 0.0;
  const double scale = (run->scatter_scale > 0.0) ? run->scatter_scale : 1.0;
  if (wtask) wtask->assign((size_t)nm * ns * (na - 1), 0.0);
  std::vector<double> sw(run->nbins, 0.0), swt(run->nbins, 0.0), sv(run->nbins, 0.0);
  std::vector<double> Sv(ns), Vv(ns), dE(ns);
  for (int64_t m = 0; m < nm; ++m) {
    for (int s = 0; s < ns; ++s) {
      double acc = 0.0, var = 0.0;
      for (int ia = 0; ia < na - 1; ++ia) {
        const int64_t task = m + nm * (s + (int64_t)ns * ia);
        const double tr = (double)counts[task] / np;
        acc += coef[ia] * tr;
        var += coef[ia] * coef[ia] * (tr * (1.0 - tr) / np);
        if (out->transmit) out->transmit[task] = tr;
      }
      if (out->transmit) out->transmit[m + nm * (s + (int64_t)ns * (na - 1))] = 0.0;
      Sv[s] = acc * dS;
      Vv[s] = var * dS * dS;
      dE[s] = 0.0;
    }
    const double mf = mc.mfp_m[m];
    double E;
    if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
      if (mf == 0.0) { E = Sv[0] * 1.0e-9; dE[0] = 1.0e-9; }
      else {
        const double sm = Sv[0] * 1.0e-9;
        E = 1.0 / (1.0 / mf + 1.0 / sm);
        dE[0] = (sm > 0.0) ? 1.0e-9 * (E * E) / (sm * sm) : 1.0e-9;
      }
    } else if (run->kind_mfp == PTG_MFP_PER_MODE) {
      E = Sv[0] * 1.0e-9;
      dE[0] = 1.0e-9;
    } else {
      const double* g = run->mfp_grid_nm;
      if (mf < g[0] * 1.0e-9) {
        E = Sv[0] * 1.0e-9 * mf / (g[0] * 1.0e-9);
        dE[0] = 1.0e-9 * mf / (g[0] * 1.0e-9);
      } else if (mf > g[ns - 1] * 1.0e-9) {
        E = Sv[ns - 1] * 1.0e-9;
        dE[ns - 1] = 1.0e-9;
      } else {
        E = Sv[ns - 1] * 1.0e-9;
        dE[ns - 1] = 1.0e-9;
        for (int s = 0; s < ns - 1; ++s) {
          if (g[s] * 1.0e-9 <= mf && mf < g[s + 1] * 1.0e-9) {
            const double ip = (mf - g[s] * 1.0e-9) / ((g[s + 1] - g[s]) * 1.0e-9);
            E = Sv[s] * 1.0e-9 * (1.0 - ip) + Sv[s + 1] * 1.0e-9 * ip;
            dE[ns - 1] = 0.0;
            dE[s] = 1.0e-9 * (1.0 - ip);
            dE[s + 1] = 1.0e-9 * ip;
            break;
          }
        }
      }
    }
    kappa += mc.K[m] * E;
    for (int s = 0; s < ns; ++s) {
      const double gk = mc.K[m] * dE[s];
      kvar += gk * gk * Vv[s];
      if (wtask)
        for (int ia = 0; ia < na - 1; ++ia)
          (*wtask)[m + nm * (s + (int64_t)ns * ia)] = gk * dS * coef[ia];
    }
    /* d E / d s through the bulk MFP mf = MFP0 / s */
    if (run->kind_mfp == PTG_MFP_MATTHIESSEN && mf > 0.0) {
      dks += mc.K[m] * (-(E * E) / (mf * scale));
    } else if (run->kind_mfp == PTG_MFP_GRID) {
      const double* g = run->mfp_grid_nm;
      double dEdm = 0.0;
      if (mf < g[0] * 1.0e-9) {
        dEdm = Sv[0] / g[0];
      } else {
        for (int s = 0; s < ns - 1; ++s)
          if (g[s] * 1.0e-9 <= mf && mf < g[s + 1] * 1.0e-9) {
            dEdm = (Sv[s + 1] - Sv[s]) / (g[s + 1] - g[s]);
            break;
          }
      }
      dks += mc.K[m] * dEdm * (-mf / scale);
    }
    if (out->emfp_nm) out->emfp_nm[m] = E * 1.0e9;
    if (run->nbins > 0 && mc.bin[m] >= 0) {
      double tm, vm = 0.0;
      if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
        tm = Sv[0] / tnorm;
        vm = Vv[0] / (tnorm * tnorm);
      } else {
        tm = E * 1.0e9 / tnorm;
        for (int s = 0; s < ns; ++s) {
          const double gk = dE[s] * 1.0e9 / tnorm;
          vm += gk * gk * Vv[s];
        }
      }
      const int b = mc.bin[m];
      sw[b] += mc.W[m];
      swt[b] += mc.W[m] * tm;
      sv[b] += mc.W[m] * mc.W[m] * vm;
    }
  }
  out->kappa = kappa;
  out->kappa_stderr = sqrt(kvar);
  if (dk_ds_an) *dk_ds_an = dks;
  for (int b = 0; b < run->nbins; ++b) {
    if (out->bin_T) out->bin_T[b] = sw[b] > 0 ? swt[b] / sw[b] : 0.0;
    if (out->bin_T_stderr) out->bin_T_stderr[b] = sw[b] > 0 ? sqrt(sv[b]) / sw[b] : 0.0;
  }
  return PTG_OK;
}


int handle_noalloc_view(ptg_handle* h, NoallocView* v) {
  if (!h || !v) return PTG_ERR_INVALID;
  v->g32 = h->g32;
  v->blob_bytes = h->blob_bytes;
  v->device = h->device;
  v->num_sms = h->num_sms;
  v->stream = h->stream;
  v->opt = h->opt;
  v->spec = &h->spec;
  v->geom = &h->geom;
  v->last = &h->last;
  return PTG_OK;
}

}  // namespace ptg

/* ========================================================================= */
extern "C" {

const char* ptg_strerror(int status) {
  switch (status) {
    case PTG_OK: return "ok";
    case PTG_ERR_INVALID: return "invalid argument or inconsistent input";
    case PTG_ERR_CUDA: return "CUDA runtime error";
    case PTG_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
    case PTG_ERR_TIMEOUT: return "a bounded device wait timed out";
    case PTG_ERR_LOST: return "lost-phonon fraction above the limit";
    case PTG_ERR_NOMEM: return "out of memory";
    case PTG_ERR_IO: return "file missing or malformed";
    case PTG_ERR_UNSUPPORTED: return "unsupported combination";
  }
  return "unknown status";
}

int ptg_create(const ptg_geometry* geom, const ptg_spectrum* spec, const ptg_options* opt,
               ptg_handle** out) {
  ptg_handle* h = nullptr;
  try {
    if (!out) return PTG_ERR_INVALID;
    *out = nullptr;
    h = ptg::alloc_should_fail() ? nullptr : new (std::nothrow) ptg_handle();
    if (!h) return PTG_ERR_NOMEM;
    memset(&h->opt, 0, sizeof(h->opt));
    if (opt) h->opt = *opt;
    memset(&h->last, 0, sizeof(h->last));
    if (h->opt.reserved != 0) { delete h; return PTG_ERR_INVALID; }
    std::string why;
    int st = ptg::copy_geometry(geom, &h->geom, &why);
    if (st == PTG_OK) st = ptg::copy_spectrum(spec, &h->spec, &why);
    if (st != PTG_OK) { delete h; return st; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || h->opt.device < 0 ||
        h->opt.device >= ndev) {
      cudaGetLastError();
      delete h;
      return PTG_ERR_NO_DEVICE;
    }
    h->device = h->opt.device;
    cudaDeviceProp prop;
    if (cudaSetDevice(h->device) != cudaSuccess ||
        cudaGetDeviceProperties(&prop, h->device) != cudaSuccess || prop.major != 10) {
      cudaGetLastError();
      delete h;
      return PTG_ERR_NO_DEVICE;
    }
    h->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return PTG_ERR_CUDA;
    }
    for (auto& e : h->ev)
      if (cudaEventCreate(&e) != cudaSuccess) { delete h; return PTG_ERR_CUDA; }
    if (cudaEventCreateWithFlags(&h->h2d_done, cudaEventDisableTiming) != cudaSuccess) {
      delete h;
      return PTG_ERR_CUDA;
    }
    st = build_geo64(h);
    if (st == PTG_OK) st = build_blob(h);
    if (st != PTG_OK) { delete h; return st; }
    *out = h;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    delete h;
    if (out) *out = nullptr;
    return PTG_ERR_NOMEM;
  } catch (...) {
    delete h;
    if (out) *out = nullptr;
    return PTG_ERR_INVALID;
  }
}

int ptg_set_spectrum(ptg_handle* h, const ptg_spectrum* spec) {
  if (!h || !spec) return PTG_ERR_INVALID;
  if (spec->nbranch != h->spec.nb || spec->nkpoint != h->spec.nk) return PTG_ERR_INVALID;
  std::string why;
  ptg::SpecSoA s;
  int st = ptg::copy_spectrum(spec, &s, &why);
  if (st != PTG_OK) return st;
  h->spec = s;
  h->g64.max_omega = h->spec.max_omega;
  return PTG_OK;
}

int ptg_get_options(const ptg_handle* h, ptg_options* out) {
  if (!h || !out) return PTG_ERR_INVALID;
  *out = h->opt;
  return PTG_OK;
}

int ptg_set_options(ptg_handle* h, const ptg_options* opt) {
  try {
    if (!h || !opt) return PTG_ERR_INVALID;
    if (opt->device != h->device) { h->last_error = "options name another device"; return PTG_ERR_INVALID; }
    if (opt->block_size != 0 && (opt->block_size < 32 || opt->block_size > 256 || opt->block_size % 32)) {
      h->last_error = "block_size must be 0 or a multiple of 32 up to 256";
      return PTG_ERR_INVALID;
    }
    if (opt->reserved != 0) { h->last_error = "ptg_options.reserved must be 0"; return PTG_ERR_INVALID; }
    const bool rebuild = opt->bvh_leaf != h->opt.bvh_leaf;
    const ptg_options old = h->opt;
    h->opt = *opt;
    if (rebuild) {
      if (cudaSetDevice(h->device) != cudaSuccess) { h->opt = old; return PTG_ERR_CUDA; }
      if (cudaStreamSynchronize(h->stream) != cudaSuccess) { h->opt = old; return PTG_ERR_CUDA; }
      const int st = build_blob(h);
      if (st != PTG_OK) {
        h->opt = old;
        build_blob(h);
        return st;
      }
    }
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

void ptg_destroy(ptg_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
}

int ptg_transmission(ptg_handle* h, double mfp_nm, int32_t nangle, int64_t np, int32_t rank,
                     int32_t nranks, uint64_t seed, int32_t precision, double* transmit,
                     double* stderr_opt) {
  try {
    ptg::NvtxRange nvtx("ptg_transmission");
    if (!h || !transmit) return PTG_ERR_INVALID;
    if (nangle < 2 || np < 1 || nranks < 1 || rank < 0 || rank >= nranks) return PTG_ERR_INVALID;
    if (precision != PTG_PREC_FP32 && precision != PTG_PREC_FP64) return PTG_ERR_INVALID;
    if (!(mfp_nm > 0.0)) return PTG_ERR_INVALID;
    const int64_t nm = (int64_t)h->spec.nb * h->spec.nk;
    const int64_t ntask = nm * (nangle - 1);
    std::vector<ptg::TaskHost> tasks(ntask);
    const double half_pi = 3.14159265358979323846 * 0.5;
    for (int64_t t = 0; t < ntask; ++t) {
      const int64_t m = t % nm, ia = t / nm;
      const double theta = 0.0 + (double)ia / (double)(nangle - 1) * half_pi;
      tasks[t] = {mfp_nm, cos(theta), sin(theta), h->spec.omega[m]};
    }
    Transport T;
    T.ntask = ntask;
    T.np = np;
    T.np_local = np_local_of(np, rank, nranks);
    if (T.np_local > 2147483647LL) return PTG_ERR_INVALID;
    T.rank = rank;
    T.nranks = nranks;
    T.seed = seed;
    T.precision = precision;
    T.tasks = &tasks;
    T.npair = h->spec.nmode();
    int st = run_transport(h, T);
    if (st != PTG_OK) return st;
    std::vector<unsigned long long> cnt(ntask);
    CU(cudaMemcpyAsync(cnt.data(), h->counts.p, sizeof(unsigned long long) * ntask,
                       cudaMemcpyDeviceToHost, h->stream));
    h->last.d2h_bytes += sizeof(unsigned long long) * ntask;
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    for (int64_t t = 0; t < nm * nangle; ++t) {
      double v = 0.0;
      if (t < ntask) v = (double)cnt[t] / (double)np;
      transmit[t] = v;
      if (stderr_opt) stderr_opt[t] = sqrt(v * (1.0 - v) / (double)np);
    }
    return check_lost(h);
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_kappa(ptg_handle* h, const ptg_run* run, ptg_kappa_out* out) {
  try {
    ptg::NvtxRange nvtx("ptg_kappa");
    if (!h || !run || !out) return PTG_ERR_INVALID;
    std::string why;
    if (!ptg::run_valid(h->spec, run, &why)) { h->last_error = why; return PTG_ERR_INVALID; }
    if (run->precision != PTG_PREC_FP32 && run->precision != PTG_PREC_FP64) return PTG_ERR_INVALID;
    const int ns = run->kind_mfp == PTG_MFP_GRID ? run->nmfp : 1;
    if (ns > 64) { h->last_error = "at most 64 grid MFPs"; return PTG_ERR_UNSUPPORTED; }
    std::vector<ptg::TaskHost> tasks;
    ptg::run_tasks(h->spec, run, &tasks);
    Transport T;
    T.ntask = (int64_t)tasks.size();
    T.np = run->np;
    T.np_local = np_local_of(run->np, run->rank, run->nranks);
    if (T.np_local > 2147483647LL) return PTG_ERR_INVALID;
    T.rank = run->rank;
    T.nranks = run->nranks;
    T.seed = run->seed;
    T.stream = run->stream;
    T.precision = run->precision;
    T.tasks = &tasks;
    T.npair = h->spec.nmode() * ns;
    int st = run_transport(h, T);
    if (st != PTG_OK) return st;
    /* FP64 reduction on the device */
    const int64_t nm = h->spec.nmode();
    ptg::ModeConst mc;
    ptg::mode_constants(h->spec, run, &mc);
    std::vector<double> coef;
    double dS = 0.0;
    ptg::simpson_weights(run->nangle, h->geom.box[0], &coef, &dS);
    const int nbins = run->nbins;
    CU(h->red_coef.ensure(sizeof(double) * coef.size()));
    CU(h->red_K.ensure(sizeof(double) * nm));
    CU(h->red_W.ensure(sizeof(double) * nm));
    CU(h->red_mfp.ensure(sizeof(double) * nm));
    CU(h->red_bin.ensure(sizeof(int) * nm));
    CU(h->red_grid.ensure(sizeof(double) * ns));
    CU(h->red_tc.ensure(sizeof(double) * nm));
    CU(h->red_kv.ensure(sizeof(double) * nm));
    CU(h->red_bw.ensure(sizeof(double) * nm));
    CU(h->red_bv.ensure(sizeof(double) * nm));
    CU(h->red_emfp.ensure(sizeof(double) * nm));
    CU(h->red_trans.ensure(sizeof(double) * nm * ns * run->nangle));
    CU(h->red_result.ensure(sizeof(double) * (2 + 3 * (size_t)nbins)));
    cudaStream_t s = h->stream;
    CU(cudaMemcpyAsync(h->red_coef.p, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(h->red_K.p, mc.K.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(h->red_W.p, mc.W.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(h->red_mfp.p, mc.mfp_m.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(h->red_bin.p, mc.bin.data(), sizeof(int) * nm, cudaMemcpyHostToDevice, s));
    if (run->kind_mfp == PTG_MFP_GRID)
      CU(cudaMemcpyAsync(h->red_grid.p, run->mfp_grid_nm, sizeof(double) * ns, cudaMemcpyHostToDevice, s));
    h->last.h2d_bytes += sizeof(double) * (coef.size() + 3 * (size_t)nm) + sizeof(int) * nm +
                         (run->kind_mfp == PTG_MFP_GRID ? sizeof(double) * ns : 0);
    ptg::ReduceIn in;
    memset(&in, 0, sizeof(in));
    in.counts = h->counts.as<const unsigned long long>();
    in.nmode = nm;
    in.nangle = run->nangle;
    in.ns = ns;
    in.kind_mfp = run->kind_mfp;
    in.nbins = nbins;
    in.np = (double)run->np;
    in.dS = dS;
    in.tnorm = 0.75 * h->geom.box[0];
    in.coef = h->red_coef.as<const double>();
    in.K = h->red_K.as<const double>();
    in.W = h->red_W.as<const double>();
    in.mfp_m = h->red_mfp.as<const double>();
    in.bin = h->red_bin.as<const int>();
    in.grid = h->red_grid.as<const double>();
    in.tc = h->red_tc.as<double>();
    in.kv = h->red_kv.as<double>();
    in.bw = h->red_bw.as<double>();
    in.bv = h->red_bv.as<double>();
    in.emfp_nm = h->red_emfp.as<double>();
    in.transmit = h->red_trans.as<double>();
    in.result = h->red_result.as<double>();
    {
      ptg::NvtxRange nvtx("ptg kappa reduction");
      CU(cudaEventRecord(h->ev[2], s));
      CU(ptg::launch_kappa_reduce(in, s));
      CU(cudaEventRecord(h->ev[3], s));
    }
    std::vector<double> res(2 + 3 * (size_t)nbins);
    CU(cudaMemcpyAsync(res.data(), h->red_result.p, sizeof(double) * res.size(), cudaMemcpyDeviceToHost, s));
    if (out->emfp_nm)
      CU(cudaMemcpyAsync(out->emfp_nm, h->red_emfp.p, sizeof(double) * nm, cudaMemcpyDeviceToHost, s));
    if (out->transmit)
      CU(cudaMemcpyAsync(out->transmit, h->red_trans.p, sizeof(double) * nm * ns * run->nangle,
                         cudaMemcpyDeviceToHost, s));
    if (out->counts)
      CU(cudaMemcpyAsync(out->counts, h->counts.p, sizeof(unsigned long long) * T.ntask,
                         cudaMemcpyDeviceToHost, s));
    h->last.d2h_bytes += sizeof(double) * res.size() + (out->emfp_nm ? sizeof(double) * nm : 0) +
                         (out->transmit ? sizeof(double) * nm * ns * run->nangle : 0) +
                         (out->counts ? sizeof(unsigned long long) * T.ntask : 0);
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    float rms = 0.f;
    CU(cudaEventElapsedTime(&rms, h->ev[2], h->ev[3]));
    h->last.reduce_ms = rms;
    h->last.launches += 2;
    out->kappa = res[0];
    out->kappa_stderr = sqrt(res[1]);
    for (int b = 0; b < nbins; ++b) {
      const double sw = res[2 + 3 * b], swt = res[3 + 3 * b], sv = res[4 + 3 * b];
      if (out->bin_T) out->bin_T[b] = sw > 0 ? swt / sw : 0.0;
      if (out->bin_T_stderr) out->bin_T_stderr[b] = sw > 0 ? sqrt(sv) / sw : 0.0;
    }
    out->flights = h->last.flights;
    out->lost = h->last.lost;
    out->samples = h->last.samples;
    out->kernel_ms = h->last.kernel_ms;
    return check_lost(h);
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_kappa_from_counts(const ptg_geometry* geom, const ptg_spectrum* spec, const ptg_run* run,
                          const uint64_t* counts, ptg_kappa_out* out) {
  try {
    if (!geom || !spec || !run || !counts || !out) return PTG_ERR_INVALID;
    ptg::SpecSoA S;
    std::string why;
    if (ptg::copy_spectrum(spec, &S, &why) != PTG_OK) return PTG_ERR_INVALID;
    if (!ptg::run_valid(S, run, &why)) return PTG_ERR_INVALID;
    return ptg::assemble_host(S, run, geom->box[0], counts, out, nullptr, nullptr);
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_trace(ptg_handle* h, const ptg_run* run, int64_t n, const uint64_t* samples,
              int64_t cap_positions, float* pos, int64_t* npos, int32_t* end_side) {
  try {
    ptg::NvtxRange nvtx("ptg_trace");
    if (!h || !run || n < 1 || !samples || !npos || !end_side) return PTG_ERR_INVALID;
    std::string why;
    if (!ptg::run_valid(h->spec, run, &why)) { h->last_error = why; return PTG_ERR_INVALID; }
    std::vector<ptg::TaskHost> tasks;
    ptg::run_tasks(h->spec, run, &tasks);
    const uint64_t total = (uint64_t)tasks.size() * (uint64_t)run->np;
    for (int64_t i = 0; i < n; ++i)
      if (samples[i] >= total) { h->last_error = "sample id beyond ntask * np"; return PTG_ERR_INVALID; }
    CU(cudaSetDevice(h->device));
    CU(h->adj_list.ensure(sizeof(unsigned long long) * n));
    CU(h->tr_npos.ensure(sizeof(long long) * n));
    CU(h->tr_end.ensure(sizeof(int) * n));
    CU(h->tr_off.ensure(sizeof(long long) * (n + 1)));
    CU(cudaMemcpyAsync(h->adj_list.p, samples, sizeof(unsigned long long) * n, cudaMemcpyHostToDevice,
                       h->stream));
    Transport T;
    T.ntask = (int64_t)tasks.size();
    T.np = run->np;
    T.np_local = 0;  /* no chunk queue: the kernel walks the replay list */
    T.seed = run->seed;
    T.stream = run->stream;
    T.precision = PTG_PREC_FP32;
    T.tasks = &tasks;
    T.mode = ptg::MODE_TRACE;
    T.alist = h->adj_list.as<const unsigned long long>();
    T.alist_n = (long long)n;
    T.trace_off = h->tr_off.as<const long long>();
    T.trace_npos = h->tr_npos.as<long long>();
    T.trace_end = h->tr_end.as<int>();
    /* pass 1: lengths and exits */
    int st = run_transport(h, T);
    if (st != PTG_OK) return st;
    std::vector<long long> cnt(n);
    std::vector<int> ends(n);
    CU(cudaMemcpyAsync(cnt.data(), h->tr_npos.p, sizeof(long long) * n, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(ends.data(), h->tr_end.p, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    long long sum = 0;
    for (int64_t i = 0; i < n; ++i) {
      npos[i] = cnt[i];
      end_side[i] = ends[i];
      sum += cnt[i];
    }
    if (!pos) return PTG_OK;
    if (sum > cap_positions) { h->last_error = "position buffer smaller than the trajectories"; return PTG_ERR_INVALID; }
    /* pass 2: the same trajectories, positions recorded at exclusive offsets */
    std::vector<long long> off(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + cnt[i];
    CU(h->tr_pos.ensure(sizeof(float) * 3 * (size_t)(sum > 0 ? sum : 1)));
    CU(cudaMemcpyAsync(h->tr_off.p, off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice,
                       h->stream));
    T.trace = h->tr_pos.as<float>();
    st = run_transport(h, T);
    if (st != PTG_OK) return st;
    CU(cudaMemcpyAsync(pos, h->tr_pos.p, sizeof(float) * 3 * (size_t)sum, cudaMemcpyDeviceToHost,
                       h->stream));
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    h->last.d2h_bytes += sizeof(float) * 3 * (size_t)sum;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_write_trace(ptg_handle* h, const ptg_run* run, int32_t particle_trace, const char* path) {
  try {
    if (!h || !run || particle_trace < 1 || !path) return PTG_ERR_INVALID;
    std::string why;
    if (!ptg::run_valid(h->spec, run, &why)) { h->last_error = why; return PTG_ERR_INVALID; }
    const uint64_t total = (uint64_t)ptg::run_ntask(h->spec, run) * (uint64_t)run->np;
    /* interval_trace of RayTrace, src/RTMCphon.f90:3373-3375 (one rank) */
    uint64_t interval = total / (uint64_t)particle_trace;
    if (interval < 1) interval = 1;
    std::vector<uint64_t> samples;
    for (uint64_t k = 0; k < (uint64_t)particle_trace && k * interval < total; ++k)
      samples.push_back(k * interval);
    const int64_t n = (int64_t)samples.size();
    std::vector<int64_t> npos(n);
    std::vector<int32_t> ends(n);
    int st = ptg_trace(h, run, n, samples.data(), 0, nullptr, npos.data(), ends.data());
    if (st != PTG_OK) return st;
    int64_t sum = 0;
    for (int64_t v : npos) sum += v;
    std::vector<float> pos(3 * (size_t)(sum > 0 ? sum : 1));
    st = ptg_trace(h, run, n, samples.data(), sum, pos.data(), npos.data(), ends.data());
    if (st != PTG_OK) return st;
    FILE* f = fopen(path, "w");
    if (!f) return PTG_ERR_IO;
    fprintf(f, "# Datatype = trace\n");
    fprintf(f, "# particle_trace = %8d\n", (int)particle_trace);
    fprintf(f, "# interval_trace = %8lld\n", (long long)interval);
    fprintf(f, "\n");
    size_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t j = 0; j < npos[i]; ++j, ++k)
        fprintf(f, " %15.8E %15.8E %15.8E\n", pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]);
      fprintf(f, "\n\n");
    }
    return fclose(f) == 0 ? PTG_OK : PTG_ERR_IO;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_adjoint(ptg_handle* h, const ptg_run* run, ptg_adjoint_out* out) {
  try {
    ptg::NvtxRange nvtx("ptg_adjoint");
    if (!h || !run || !out) return PTG_ERR_INVALID;
    std::string why;
    if (!ptg::run_valid(h->spec, run, &why)) { h->last_error = why; return PTG_ERR_INVALID; }
    const int ns = run->kind_mfp == PTG_MFP_GRID ? run->nmfp : 1;
    if (ns > 64) return PTG_ERR_UNSUPPORTED;
    std::vector<ptg::TaskHost> tasks;
    ptg::run_tasks(h->spec, run, &tasks);
    const int64_t ntask = (int64_t)tasks.size();
    const int nsurf = h->geom.nsurf();
    const unsigned long long cap = 1ull << 31;  /* listed ids: at most every sample of the run */
    CU(cudaSetDevice(h->device));
    /* 1. forward pass that lists the samples leaving through x+ */
    Transport T;
    T.ntask = ntask;
    T.np = run->np;
    T.np_local = np_local_of(run->np, run->rank, run->nranks);
    if (T.np_local > 2147483647LL) return PTG_ERR_INVALID;
    T.rank = run->rank;
    T.nranks = run->nranks;
    T.seed = run->seed;
    T.stream = run->stream;
    T.precision = PTG_PREC_FP32;
    T.tasks = &tasks;
    T.npair = h->spec.nmode() * ns;
    T.mode = ptg::MODE_LIST;
    const unsigned long long total = (unsigned long long)ntask * (unsigned long long)T.np_local;
    T.tlist_cap = total < cap ? total : cap;
    CU(h->adj_list.ensure(sizeof(unsigned long long) * (T.tlist_cap ? T.tlist_cap : 1)));
    T.tlist = h->adj_list.as<unsigned long long>();
    int st = run_transport(h, T);
    if (st != PTG_OK) return st;
    std::vector<uint64_t> counts(ntask);
    CU(cudaMemcpyAsync(counts.data(), h->counts.p, sizeof(uint64_t) * ntask, cudaMemcpyDeviceToHost,
                       h->stream));
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    const double fwd_ms = h->last.kernel_ms;
    const uint64_t fwd_flights = h->last.flights;
    const unsigned long long nlist = h->list_n;
    if (nlist > T.tlist_cap) { h->last_error = "more than 2^31 transmitted samples"; return PTG_ERR_UNSUPPORTED; }
    /* 2. kappa and d kappa / d T_task on the host */
    ptg_kappa_out ko;
    memset(&ko, 0, sizeof(ko));
    std::vector<double> wtask;
    double dks_an = 0.0;
    st = ptg::assemble_host(h->spec, run, h->geom.box[0], counts.data(), &ko, &wtask, &dks_an);
    if (st != PTG_OK) return st;
    std::vector<float> wsample(ntask);
    for (int64_t t = 0; t < ntask; ++t) wsample[t] = (float)(wtask[t] / (double)run->np);
    CU(h->adj_w.ensure(sizeof(float) * ntask));
    CU(cudaMemcpyAsync(h->adj_w.p, wsample.data(), sizeof(float) * ntask, cudaMemcpyHostToDevice,
                       h->stream));
    const size_t nacc = (size_t)ptg::kAdjBatches * (nsurf + 1);
    CU(h->adj_acc.ensure(sizeof(double) * nacc));
    CU(cudaMemsetAsync(h->adj_acc.p, 0, sizeof(double) * nacc, h->stream));
    /* 3. replay of the listed samples with the score accumulation */
    T.mode = ptg::MODE_ADJOINT;
    T.tlist = nullptr;
    T.tlist_cap = 0;
    T.alist = h->adj_list.as<const unsigned long long>();
    T.alist_n = (long long)nlist;
    T.wsample = h->adj_w.as<const float>();
    T.adj = h->adj_acc.as<double>();
    st = run_transport(h, T);
    if (st != PTG_OK) return st;
    std::vector<double> acc(nacc);
    CU(cudaMemcpyAsync(acc.data(), h->adj_acc.p, sizeof(double) * nacc, cudaMemcpyDeviceToHost,
                       h->stream));
    st = finish_stats(h);
    if (st != PTG_OK) return st;
    /* 4. batch sums and standard errors */
    const int B = ptg::kAdjBatches;
    auto reduce = [&](int col, double* mean_total, double* se) {
      double sum = 0.0, sq = 0.0;
      for (int b = 0; b < B; ++b) sum += acc[(size_t)b * (nsurf + 1) + col];
      const double mb = sum / B;
      for (int b = 0; b < B; ++b) {
        const double d = acc[(size_t)b * (nsurf + 1) + col] - mb;
        sq += d * d;
      }
      *mean_total = sum;
      *se = sqrt((double)B * sq / (B - 1));
    };
    for (int k = 0; k < nsurf; ++k) {
      double v, e;
      reduce(k, &v, &e);
      const double p = h->geom.specularity[k];
      const bool interior = p > 0.0 && p < 1.0;
      if (out->dk_dp) out->dk_dp[k] = interior ? v : NAN;
      if (out->dk_dp_stderr) out->dk_dp_stderr[k] = interior ? e : NAN;
    }
    double vs, es;
    reduce(nsurf, &vs, &es);
    out->dk_dscale = (run->kind_mfp == PTG_MFP_PER_MODE ? vs : 0.0) + dks_an;
    out->dk_dscale_stderr = run->kind_mfp == PTG_MFP_PER_MODE ? es : 0.0;
    out->kappa = ko.kappa;
    out->kappa_stderr = ko.kappa_stderr;
    out->flights = fwd_flights + h->last.flights;
    out->replayed = nlist;
    out->mismatched = h->mismatch;
    out->kernel_ms = fwd_ms + h->last.kernel_ms;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

int ptg_check_report(int32_t device, int64_t* violations, int32_t* first_code, int32_t* first_index,
                     int32_t reset) {
  if (!violations || !first_code || !first_index) return PTG_ERR_INVALID;
  long long n = 0;
  int code = 0, index = 0;
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return PTG_ERR_NO_DEVICE; }
  const cudaError_t e = ptg::check_report(&n, &code, &index, reset != 0);
  if (e == cudaErrorNotSupported) return PTG_ERR_UNSUPPORTED;
  if (e != cudaSuccess) { cudaGetLastError(); return PTG_ERR_CUDA; }
  *violations = n;
  *first_code = code;
  *first_index = index;
  return PTG_OK;
}

int ptg_last_stats(const ptg_handle* h, ptg_stats* st) {
  if (!h || !st) return PTG_ERR_INVALID;
  *st = h->last;
  return PTG_OK;
}

int ptg_replay_task(ptg_handle* h, const ptg_run* run, int64_t task, int32_t* end_side,
                    uint32_t* flights, double* final_pos) {
  if (!h || !run || !end_side || !flights || !final_pos) return PTG_ERR_INVALID;
  std::string why;
  if (!ptg::run_valid(h->spec, run, &why)) return PTG_ERR_INVALID;
  std::vector<ptg::TaskHost> tasks;
  ptg::run_tasks(h->spec, run, &tasks);
  if (task < 0 || task >= (int64_t)tasks.size()) return PTG_ERR_INVALID;
  const int64_t npl = np_local_of(run->np, run->rank, run->nranks);
  CU(cudaSetDevice(h->device));
  const int64_t ntask = (int64_t)tasks.size();
  std::vector<ptg::Task64> t64(ntask);
  for (int64_t i = 0; i < ntask; ++i) t64[i] = {tasks[i].lambda, tasks[i].cth, tasks[i].sth, tasks[i].omega};
  DevBuf dt, de, df, dp, dc, dl, ds;
  int st = PTG_OK;
  do {
    if (dt.ensure(sizeof(ptg::Task64) * ntask) || de.ensure(sizeof(int) * npl) ||
        df.ensure(sizeof(unsigned) * npl) || dp.ensure(sizeof(double) * 3 * npl) ||
        dc.ensure(sizeof(unsigned long long) * ntask) || dl.ensure(sizeof(unsigned long long) * ntask) ||
        ds.ensure(sizeof(unsigned long long) * 4)) { st = PTG_ERR_CUDA; break; }
    cudaMemcpy(dt.p, t64.data(), sizeof(ptg::Task64) * ntask, cudaMemcpyHostToDevice);
    cudaMemset(dc.p, 0, sizeof(unsigned long long) * ntask);
    cudaMemset(dl.p, 0, sizeof(unsigned long long) * ntask);
    cudaMemset(ds.p, 0, sizeof(unsigned long long) * 4);
    ptg::Run64 r;
    memset(&r, 0, sizeof(r));
    r.task = dt.as<const ptg::Task64>();
    r.ntask = ntask;
    r.np = run->np;
    r.np_local = npl;
    r.rank = run->rank;
    r.nranks = run->nranks;
    r.k0 = (uint32_t)run->seed;
    r.k1 = (uint32_t)(run->seed >> 32);
    r.c1 = ((uint32_t)run->stream) << 8;
    r.max_flights = h->opt.max_flights > 0 ? h->opt.max_flights : 10000000LL;
    r.ref_quirks = h->opt.ref_quirks;
    r.counts = dc.as<unsigned long long>();
    r.lost = dl.as<unsigned long long>();
    r.stats = ds.as<unsigned long long>();
    r.replay_task = task;
    r.end_side = de.as<int>();
    r.flights = df.as<unsigned>();
    r.final_pos = dp.as<double>();
    if (ptg::launch_plain_fp64(h->g64, r, h->stream, nullptr, nullptr) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) { st = PTG_ERR_CUDA; break; }
    cudaMemcpy(end_side, de.p, sizeof(int) * npl, cudaMemcpyDeviceToHost);
    cudaMemcpy(flights, df.p, sizeof(unsigned) * npl, cudaMemcpyDeviceToHost);
    if (cudaMemcpy(final_pos, dp.p, sizeof(double) * 3 * npl, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = PTG_ERR_CUDA;
  } while (0);
  DevBuf* all[] = {&dt, &de, &df, &dp, &dc, &dl, &ds};
  for (DevBuf* b : all) b->release();
  return st;
}

}  // extern "C"
