/*
 * batch.cpp - many geometries in one persistent launch, replayed as a CUDA
 * graph (ptg_batch_*).
 *
 * Every geometry keeps the sample numbering, seed and stream of a single-
 * geometry ptg_kappa run (the reference's TransmissionFunction per structure,
 * src/RTMCphon.f90:1544-1604), so a batched run gives each geometry exactly
 * the transmitted counts of its own run.  The work queue spans all
 * geometries' (mode, angle) tasks, longest expected trajectories first, so
 * geometries with very uneven sample counts and mean free paths share the
 * GPU without a tail per geometry.  Set-up builds every table once; each
 * ptg_batch_run replays one graph: clear the tallies, the batched transport
 * kernel, the batched FP64 kappa reduction (effectiveMFP + the kappa sum,
 * :2418-2451, :2645-2755) and the copy of the results to pinned memory.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "kernels.h"
#include "ptg_internal.h"

namespace {

struct Dev {
  void* p = nullptr;
  cudaError_t alloc(size_t bytes) {
    if (ptg::alloc_should_fail()) return cudaErrorMemoryAllocation;
    return cudaMalloc(&p, bytes < 256 ? 256 : bytes);
  }
  ~Dev() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

}  // namespace

struct ptg_batch {
  int device = 0, num_sms = 0, ngeo = 0, nbins = 0;
  int64_t ntask_per_geo = 0, nmode = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  Dev blob, geos, tasks, task_geo, chunks, counts, lost, stats, queue;
  Dev coef, K, W, mfp, bin, grid, tc, kv, bw, bv, emfp, result, np_geo, dS_geo, tnorm_geo;
  double* host_result = nullptr;              /* pinned */
  unsigned long long* host_stats = nullptr;   /* pinned */
  int launch_grid = 0;
  bool bvh = false;   /* a BVH or capped cylinders: the kernel built for them */
  /* what the per-geometry adjoint needs besides the forward's tables */
  ptg::SpecSoA spec;
  ptg_run run;
  std::vector<double> mfp_grid;               /* run.mfp_grid_nm points here */
  ptg::RunF32 r;                              /* the forward's kernel arguments */
  std::vector<int> nsurf, adj_base;
  std::vector<std::vector<double>> specularity;
  std::vector<double> box_x;
  std::vector<int64_t> np;
  Dev adj_list, adj_w, adj_acc;
  size_t adj_list_cap = 0, adj_acc_n = 0;
  ~ptg_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (host_result) cudaFreeHost(host_result);
    if (host_stats) cudaFreeHost(host_stats);
    if (stream) cudaStreamDestroy(stream);
  }
};

#define BCU(x)                                                                \
  do {                                                                        \
    const cudaError_t e_ = (x);                                               \
    if (e_ != cudaSuccess) {                                                  \
      cudaGetLastError();                                                     \
      delete b;                                                               \
      b = nullptr;                                                            \
      return e_ == cudaErrorMemoryAllocation ? PTG_ERR_NOMEM : PTG_ERR_CUDA;  \
    }                                                                         \
  } while (0)

extern "C" int ptg_batch_create(const ptg_batch_item* items, int32_t nitems,
                                const ptg_spectrum* spec, const ptg_run* run,
                                const ptg_options* opt, ptg_batch** out) {
  ptg_batch* b = nullptr;
  try {
    if (!items || nitems < 1 || nitems > 65535 || !spec || !run || !out) return PTG_ERR_INVALID;
    *out = nullptr;
    std::string why;
    ptg::SpecSoA S;
    if (ptg::copy_spectrum(spec, &S, &why) != PTG_OK) return PTG_ERR_INVALID;
    if (!ptg::run_valid(S, run, &why)) return PTG_ERR_INVALID;
    const int ns = run->kind_mfp == PTG_MFP_GRID ? run->nmfp : 1;
    if (ns > 64) return PTG_ERR_UNSUPPORTED;
    ptg_options o;
    memset(&o, 0, sizeof(o));
    if (opt) o = *opt;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || o.device < 0 || o.device >= ndev) {
      cudaGetLastError();
      return PTG_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaSetDevice(o.device) != cudaSuccess ||
        cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major != 10) {
      cudaGetLastError();
      return PTG_ERR_NO_DEVICE;
    }
    b = ptg::alloc_should_fail() ? nullptr : new (std::nothrow) ptg_batch();
    if (!b) return PTG_ERR_NOMEM;
    b->device = o.device;
    b->num_sms = prop.multiProcessorCount;
    b->ngeo = nitems;
    b->nbins = run->nbins;
    b->nmode = S.nmode();
  
    /* per-geometry blobs, descriptors and tasks */
    std::vector<ptg::TaskHost> tasks;
    ptg::run_tasks(S, run, &tasks);
    const int64_t ntg = (int64_t)tasks.size();
    b->ntask_per_geo = ntg;
    std::vector<float4> all_blob;
    std::vector<size_t> blob_off(nitems);
    std::vector<ptg::GeoEntry> entries(nitems);
    std::vector<double> np_geo(nitems), dS_geo(nitems), tnorm_geo(nitems);
    std::vector<double> coef;
    for (int g = 0; g < nitems; ++g) {
      const ptg_batch_item& it = items[g];
      if (it.np < 1 || it.stream < 0 || it.stream >= (1 << 24)) { delete b; return PTG_ERR_INVALID; }
      ptg::GeomSoA G;
      if (ptg::copy_geometry(it.geom, &G, &why) != PTG_OK) { delete b; return PTG_ERR_INVALID; }
      std::vector<float4> blob;
      ptg::BlobLayout L;
      if (ptg::blob_from_geometry(G, o.bvh_leaf, &blob, &L, &why) != PTG_OK) { delete b; return PTG_ERR_INVALID; }
      blob_off[g] = all_blob.size();
      all_blob.insert(all_blob.end(), blob.begin(), blob.end());
      ptg::GeoEntry& e = entries[g];
      memset(&e, 0, sizeof(e));
      e.lay = L;
      if (L.nbvh > 0 || L.ncap > 0) b->bvh = true;
      for (int d = 0; d < 3; ++d) e.box[d] = (float)G.box[d];
      e.scope[0] = (float)G.scope[0];
      e.scope[1] = (float)G.scope[1];
      const double smax = std::max(G.box[0], std::max(G.box[1], G.box[2]));
      const double smin = std::min(G.box[0], std::min(G.box[1], G.box[2]));
      e.eps = (float)(smax * (1.0 / 1048576.0));
      e.fast_lambda_max = (float)(0.1 * smin);
      for (int f = 0; f < 6; ++f)
        if (G.face_kind[f] == PTG_FACE_PERIODIC) e.periodic_mask |= 1 << f;
      e.kind_grain = G.kind_grain;
      e.igrain_fill = G.igrain_fill;
      e.nmaterial = G.nmaterial;
      e.np = it.np;
      e.k0 = (uint32_t)it.seed;
      e.k1 = (uint32_t)(it.seed >> 32);
      e.c1 = ((uint32_t)it.stream) << 8;
      e.task_base = (int)(g * ntg);
      e.nsurf = G.nsurf();
      e.adj_base = (int)b->adj_acc_n;
      b->adj_base.push_back(e.adj_base);
      b->nsurf.push_back(e.nsurf);
      b->specularity.push_back(G.specularity);
      b->box_x.push_back(G.box[0]);
      b->np.push_back(it.np);
      b->adj_acc_n += (size_t)ptg::kAdjBatches * (size_t)(e.nsurf + 1);
      if (b->adj_acc_n > 2147483647ull) { delete b; return PTG_ERR_UNSUPPORTED; }
      np_geo[g] = (double)it.np;
      double dS;
      ptg::simpson_weights(run->nangle, G.box[0], &coef, &dS);
      dS_geo[g] = dS;
      tnorm_geo[g] = 0.75 * G.box[0];
    }
    if ((int64_t)nitems * ntg > 2147483647LL) { delete b; return PTG_ERR_UNSUPPORTED; }
    std::vector<float4> t32((size_t)nitems * ntg);
    std::vector<int> task_geo((size_t)nitems * ntg);
    struct Order { double lam; int64_t t; };
    std::vector<Order> order;
    for (int g = 0; g < nitems; ++g) {
      for (int64_t t = 0; t < ntg; ++t) {
        const ptg::TaskHost& th = tasks[t];
        float lam = th.lambda == 1.0e10 ? INFINITY : (float)th.lambda;
        if (!(th.lambda > 0.0)) lam = 0.0f;
        const int64_t gt = g * ntg + t;
        t32[gt] = make_float4(lam, (float)th.cth, (float)th.sth, (float)(th.omega / S.max_omega));
        task_geo[gt] = g;
        if (th.lambda > 0.0) order.push_back({th.lambda, gt});
      }
    }
    std::stable_sort(order.begin(), order.end(), [](const Order& a, const Order& c) { return a.lam < c.lam; });
    const int64_t csz = o.chunk > 0 ? o.chunk : 64;
    std::vector<int4> chunks;
    for (const Order& od : order) {
      const int g = task_geo[od.t];
      const int64_t npl = items[g].np > run->rank ? (items[g].np - run->rank + run->nranks - 1) / run->nranks : 0;
      if (npl > 2147483647LL) { delete b; return PTG_ERR_INVALID; }
      for (int64_t j = 0; j < npl; j += csz)
        chunks.push_back(make_int4((int)od.t, (int)j, (int)std::min(csz, npl - j), 0));
    }
    if (chunks.size() > 2147483647ull) { delete b; return PTG_ERR_UNSUPPORTED; }
  
    /* device buffers */
    const size_t ntot = (size_t)nitems * ntg;
    const size_t nm = (size_t)b->nmode;
    const size_t nres = (size_t)nitems * (2 + 3 * (size_t)b->nbins);
    ptg::ModeConst mc;
    ptg::mode_constants(S, run, &mc);
    BCU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCU(cudaEventCreate(&b->ev0));
    BCU(cudaEventCreate(&b->ev1));
    BCU(b->blob.alloc(all_blob.size() * 16));
    for (int g = 0; g < nitems; ++g) entries[g].blob = b->blob.as<const float4>() + blob_off[g];
    BCU(b->geos.alloc(sizeof(ptg::GeoEntry) * nitems));
    BCU(b->tasks.alloc(sizeof(float4) * ntot));
    BCU(b->task_geo.alloc(sizeof(int) * ntot));
    BCU(b->chunks.alloc(sizeof(int4) * (chunks.size() + 1)));
    BCU(b->counts.alloc(sizeof(unsigned long long) * ntot));
    BCU(b->lost.alloc(sizeof(unsigned long long) * ntot));
    BCU(b->stats.alloc(sizeof(unsigned long long) * ptg::kStatSlots));
    BCU(b->queue.alloc(sizeof(int) * 8));
    BCU(b->coef.alloc(sizeof(double) * coef.size()));
    BCU(b->K.alloc(sizeof(double) * nm));
    BCU(b->W.alloc(sizeof(double) * nm));
    BCU(b->mfp.alloc(sizeof(double) * nm));
    BCU(b->bin.alloc(sizeof(int) * nm));
    BCU(b->grid.alloc(sizeof(double) * ns));
    BCU(b->tc.alloc(sizeof(double) * nm * nitems));
    BCU(b->kv.alloc(sizeof(double) * nm * nitems));
    BCU(b->bw.alloc(sizeof(double) * nm * nitems));
    BCU(b->bv.alloc(sizeof(double) * nm * nitems));
    BCU(b->emfp.alloc(sizeof(double) * nm * nitems));
    BCU(b->result.alloc(sizeof(double) * nres));
    BCU(b->np_geo.alloc(sizeof(double) * nitems));
    BCU(b->dS_geo.alloc(sizeof(double) * nitems));
    BCU(b->tnorm_geo.alloc(sizeof(double) * nitems));
    BCU(cudaMallocHost(&b->host_result, sizeof(double) * nres));
    BCU(cudaMallocHost(&b->host_stats, sizeof(unsigned long long) * 16));
    BCU(cudaMemcpy(b->blob.p, all_blob.data(), all_blob.size() * 16, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->geos.p, entries.data(), sizeof(ptg::GeoEntry) * nitems, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->tasks.p, t32.data(), sizeof(float4) * ntot, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->task_geo.p, task_geo.data(), sizeof(int) * ntot, cudaMemcpyHostToDevice));
    if (!chunks.empty())
      BCU(cudaMemcpy(b->chunks.p, chunks.data(), sizeof(int4) * chunks.size(), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->coef.p, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->K.p, mc.K.data(), sizeof(double) * nm, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->W.p, mc.W.data(), sizeof(double) * nm, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->mfp.p, mc.mfp_m.data(), sizeof(double) * nm, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->bin.p, mc.bin.data(), sizeof(int) * nm, cudaMemcpyHostToDevice));
    if (run->kind_mfp == PTG_MFP_GRID)
      BCU(cudaMemcpy(b->grid.p, run->mfp_grid_nm, sizeof(double) * ns, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->np_geo.p, np_geo.data(), sizeof(double) * nitems, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->dS_geo.p, dS_geo.data(), sizeof(double) * nitems, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->tnorm_geo.p, tnorm_geo.data(), sizeof(double) * nitems, cudaMemcpyHostToDevice));
  
    /* kernel arguments */
    ptg::RunF32 r;
    memset(&r, 0, sizeof(r));
    r.task = b->tasks.as<const float4>();
    r.chunk = b->chunks.as<const int4>();
    r.nchunk = (int32_t)chunks.size();
    r.rank = run->rank;
    r.nranks = run->nranks;
    const int64_t maxf = o.max_flights > 0 ? o.max_flights : 10000000LL;
    r.max_flights = (uint32_t)std::min<int64_t>(maxf, 4294967295LL);
    r.ref_quirks = o.ref_quirks;
    const int rt = o.regen_threshold > 0 ? o.regen_threshold : ptg::kDefaultRegen;
    r.regen_threshold = rt > 32 ? 32 : rt;
    r.fast_steps = (o.tune_flags & 1) ? 0 : (o.fast_steps > 0 ? o.fast_steps : ptg::kDefaultFastSteps);
    r.counts = b->counts.as<unsigned long long>();
    r.lost = b->lost.as<unsigned long long>();
    r.stats = b->stats.as<unsigned long long>();
    r.queue = b->queue.as<int>();
    r.geos = b->geos.as<const ptg::GeoEntry>();
    r.task_geo = b->task_geo.as<const int>();
    ptg::ReduceBatchIn rb;
    memset(&rb, 0, sizeof(rb));
    rb.base.counts = b->counts.as<const unsigned long long>();
    rb.base.nmode = b->nmode;
    rb.base.nangle = run->nangle;
    rb.base.ns = ns;
    rb.base.kind_mfp = run->kind_mfp;
    rb.base.nbins = run->nbins;
    rb.base.coef = b->coef.as<const double>();
    rb.base.K = b->K.as<const double>();
    rb.base.W = b->W.as<const double>();
    rb.base.mfp_m = b->mfp.as<const double>();
    rb.base.bin = b->bin.as<const int>();
    rb.base.grid = b->grid.as<const double>();
    rb.base.tc = b->tc.as<double>();
    rb.base.kv = b->kv.as<double>();
    rb.base.bw = b->bw.as<double>();
    rb.base.bv = b->bv.as<double>();
    rb.base.emfp_nm = b->emfp.as<double>();
    rb.base.result = b->result.as<double>();
    rb.ngeo = nitems;
    rb.ntask_per_geo = ntg;
    rb.np_geo = b->np_geo.as<const double>();
    rb.dS_geo = b->dS_geo.as<const double>();
    rb.tnorm_geo = b->tnorm_geo.as<const double>();
    b->r = r;
    b->spec = S;
    b->run = *run;
    if (run->kind_mfp == PTG_MFP_GRID) b->mfp_grid.assign(run->mfp_grid_nm, run->mfp_grid_nm + ns);
    b->run.mfp_grid_nm = b->mfp_grid.empty() ? nullptr : b->mfp_grid.data();
    int bps = 0;
    BCU(ptg::persistent_batch_occupancy(256, &bps, b->bvh));
    if (o.blocks_per_sm > 0 && o.blocks_per_sm < bps) bps = o.blocks_per_sm;
    if (bps < 1) bps = 1;
    b->launch_grid = b->num_sms * bps;
  
    /* capture: clear tallies, transport, reduction, results to pinned memory */
    const unsigned long long init[16] = {0, 0, 0, 0, 0, ~0ull, ~0ull, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    static_assert(sizeof(init) == 16 * sizeof(unsigned long long), "stats layout");
    unsigned long long* dstats = b->stats.as<unsigned long long>();
    BCU(cudaMemcpy(b->host_stats, init, sizeof(init), cudaMemcpyHostToHost));
    BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaMemsetAsync(b->counts.p, 0, sizeof(unsigned long long) * ntot, b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->lost.p, 0, sizeof(unsigned long long) * ntot, b->stream);
    if (ce == cudaSuccess)
      ce = cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * ptg::kStatSlots, b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(dstats + 5, 0xFF, sizeof(unsigned long long) * 2, b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->queue.p, 0, sizeof(int) * 8, b->stream);
    if (ce == cudaSuccess && r.nchunk > 0) ce = ptg::launch_persistent_batch(r, b->launch_grid, 256, b->stream, b->bvh);
    if (ce == cudaSuccess) ce = ptg::launch_kappa_reduce_batch(rb, b->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(b->host_result, b->result.p, sizeof(double) * nres, cudaMemcpyDeviceToHost,
                           b->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(b->host_stats, dstats, sizeof(unsigned long long) * 16,
                           cudaMemcpyDeviceToHost, b->stream);
    cudaGraph_t gph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &gph);
    b->graph = gph;
    if (ce != cudaSuccess || ee != cudaSuccess || !gph) { cudaGetLastError(); delete b; return PTG_ERR_CUDA; }
    BCU(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = b;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    delete b;
    if (out) *out = nullptr;
    return PTG_ERR_NOMEM;
  } catch (...) {
    delete b;
    if (out) *out = nullptr;
    return PTG_ERR_INVALID;
  }
}

extern "C" int ptg_batch_run(ptg_batch* b, ptg_batch_out* out) {
  try {
    ptg::NvtxRange nvtx("ptg_batch_run");
    if (!b || !out) return PTG_ERR_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return PTG_ERR_CUDA;
    if (cudaEventRecord(b->ev0, b->stream) != cudaSuccess ||
        cudaGraphLaunch(b->exec, b->stream) != cudaSuccess ||
        cudaEventRecord(b->ev1, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
      return PTG_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    const int nb = b->nbins;
    for (int g = 0; g < b->ngeo; ++g) {
      const double* rg = b->host_result + (size_t)g * (2 + 3 * nb);
      if (out->kappa) out->kappa[g] = rg[0];
      if (out->kappa_stderr) out->kappa_stderr[g] = sqrt(rg[1]);
      for (int k = 0; k < nb; ++k) {
        const double sw = rg[2 + 3 * k], swt = rg[3 + 3 * k], sv = rg[4 + 3 * k];
        if (out->bin_T) out->bin_T[(size_t)g * nb + k] = sw > 0 ? swt / sw : 0.0;
        if (out->bin_T_stderr) out->bin_T_stderr[(size_t)g * nb + k] = sw > 0 ? sqrt(sv) / sw : 0.0;
      }
    }
    if (out->counts &&
        cudaMemcpy(out->counts, b->counts.p, sizeof(unsigned long long) * b->ngeo * b->ntask_per_geo,
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return PTG_ERR_CUDA;
    out->flights = b->host_stats[0];
    out->lost = b->host_stats[1];
    out->samples = b->host_stats[3];
    out->graph_ms = ms;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

/* One batched transport launch outside the graph (list or adjoint mode):
   clears the tallies, statistics and queue, launches, waits; *ms receives
   its device time and st its statistics. */
static int batch_launch(ptg_batch* b, const ptg::RunF32& r, int mode, unsigned long long* st,
                        float* ms) {
  const size_t ntot = (size_t)b->ngeo * (size_t)b->ntask_per_geo;
  unsigned long long* dstats = b->stats.as<unsigned long long>();
  int bps = 0;
  if (ptg::persistent_batch_occupancy(256, &bps, b->bvh, mode) != cudaSuccess) return PTG_ERR_CUDA;
  if (bps < 1) bps = 1;
  if (cudaMemsetAsync(b->counts.p, 0, sizeof(unsigned long long) * ntot, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->lost.p, 0, sizeof(unsigned long long) * ntot, b->stream) != cudaSuccess ||
      cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * ptg::kStatSlots, b->stream) != cudaSuccess ||
      cudaMemsetAsync(dstats + 5, 0xFF, sizeof(unsigned long long) * 2, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->queue.p, 0, sizeof(int) * 8, b->stream) != cudaSuccess ||
      cudaEventRecord(b->ev0, b->stream) != cudaSuccess)
    return PTG_ERR_CUDA;
  const bool work = mode == ptg::MODE_ADJOINT ? r.alist_n > 0 : r.nchunk > 0;
  if (work && ptg::launch_persistent_batch(r, b->num_sms * bps, 256, b->stream, b->bvh, mode) != cudaSuccess)
    return PTG_ERR_CUDA;
  if (cudaEventRecord(b->ev1, b->stream) != cudaSuccess ||
      cudaMemcpyAsync(st, dstats, sizeof(unsigned long long) * ptg::kStatSlots, cudaMemcpyDeviceToHost,
                      b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return PTG_ERR_CUDA;
  *ms = 0.f;
  cudaEventElapsedTime(ms, b->ev0, b->ev1);
  return PTG_OK;
}

extern "C" int ptg_batch_adjoint(ptg_batch* b, ptg_batch_adjoint_out* out) {
  try {
    ptg::NvtxRange nvtx("ptg_batch_adjoint");
    if (!b || !out) return PTG_ERR_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return PTG_ERR_CUDA;
    const int64_t ntg = b->ntask_per_geo;
    const size_t ntot = (size_t)b->ngeo * (size_t)ntg;
    /* 1. forward pass over all geometries that lists the transmitted samples */
    unsigned long long total = 0;
    for (int g = 0; g < b->ngeo; ++g) {
      const int64_t npl = b->np[g] > b->run.rank
                              ? (b->np[g] - b->run.rank + b->run.nranks - 1) / b->run.nranks : 0;
      total += (unsigned long long)ntg * (unsigned long long)npl;
    }
    /* room for every sample of the run (at most 2^31 ids, 16 GB) */
  const unsigned long long cap = std::min<unsigned long long>(total, 1ull << 31);
    if (b->adj_list_cap < cap || !b->adj_list.p) {
      if (b->adj_list.p) { cudaFree(b->adj_list.p); b->adj_list.p = nullptr; }
      if (b->adj_list.alloc(sizeof(unsigned long long) * (cap ? cap : 1)) != cudaSuccess) return PTG_ERR_NOMEM;
      b->adj_list_cap = cap;
    }
    if (!b->adj_w.p && b->adj_w.alloc(sizeof(float) * ntot) != cudaSuccess) return PTG_ERR_NOMEM;
    if (!b->adj_acc.p && b->adj_acc.alloc(sizeof(double) * b->adj_acc_n) != cudaSuccess) return PTG_ERR_NOMEM;
    ptg::RunF32 r = b->r;
    r.tlist = b->adj_list.as<unsigned long long>();
    r.tlist_cap = cap;
    unsigned long long st[ptg::kStatSlots];
    float fwd_ms = 0.f, rep_ms = 0.f;
    int rc = batch_launch(b, r, ptg::MODE_LIST, st, &fwd_ms);
    if (rc != PTG_OK) return rc;
    const unsigned long long nlist = st[10];
    if (nlist > cap) return PTG_ERR_UNSUPPORTED;
    const uint64_t fwd_flights = st[0];
    std::vector<uint64_t> counts(ntot);
    if (cudaMemcpy(counts.data(), b->counts.p, sizeof(uint64_t) * ntot, cudaMemcpyDeviceToHost) != cudaSuccess)
      return PTG_ERR_CUDA;
    /* 2. every geometry's kappa and d kappa / d T_task on the host */
    std::vector<float> wsample(ntot);
    std::vector<double> dks_an(b->ngeo, 0.0), wtask;
    for (int g = 0; g < b->ngeo; ++g) {
      ptg_run rg = b->run;
      rg.np = b->np[g];
      ptg_kappa_out ko;
      memset(&ko, 0, sizeof(ko));
      rc = ptg::assemble_host(b->spec, &rg, b->box_x[g], counts.data() + (size_t)g * ntg, &ko, &wtask,
                              &dks_an[g]);
      if (rc != PTG_OK) return rc;
      if (out->kappa) out->kappa[g] = ko.kappa;
      if (out->kappa_stderr) out->kappa_stderr[g] = ko.kappa_stderr;
      for (int64_t t = 0; t < ntg; ++t)
        wsample[(size_t)g * ntg + t] = (float)(wtask[t] / (double)b->np[g]);
    }
    if (cudaMemcpyAsync(b->adj_w.p, wsample.data(), sizeof(float) * ntot, cudaMemcpyHostToDevice,
                        b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->adj_acc.p, 0, sizeof(double) * b->adj_acc_n, b->stream) != cudaSuccess)
      return PTG_ERR_CUDA;
    /* 3. replay of every listed sample, scores into its geometry's slice */
    r = b->r;
    r.alist = b->adj_list.as<const unsigned long long>();
    r.alist_n = (long long)nlist;
    r.wsample = b->adj_w.as<const float>();
    r.adj = b->adj_acc.as<double>();
    rc = batch_launch(b, r, ptg::MODE_ADJOINT, st, &rep_ms);
    if (rc != PTG_OK) return rc;
    std::vector<double> acc(b->adj_acc_n);
    if (cudaMemcpy(acc.data(), b->adj_acc.p, sizeof(double) * b->adj_acc_n, cudaMemcpyDeviceToHost) !=
        cudaSuccess)
      return PTG_ERR_CUDA;
    /* 4. batch sums and standard errors per geometry */
    const int B = ptg::kAdjBatches;
    size_t rec = 0;
    for (int g = 0; g < b->ngeo; ++g) {
      const int ns = b->nsurf[g];
      const double* a = acc.data() + b->adj_base[g];
      auto reduce = [&](int col, double* total_v, double* se) {
        double sum = 0.0, sq = 0.0;
        for (int k = 0; k < B; ++k) sum += a[(size_t)k * (ns + 1) + col];
        const double mb = sum / B;
        for (int k = 0; k < B; ++k) {
          const double d = a[(size_t)k * (ns + 1) + col] - mb;
          sq += d * d;
        }
        *total_v = sum;
        *se = sqrt((double)B * sq / (B - 1));
      };
      for (int k = 0; k < ns; ++k, ++rec) {
        double v, e;
        reduce(k, &v, &e);
        const double p = b->specularity[g][k];
        const bool interior = p > 0.0 && p < 1.0;
        if (out->dk_dp) out->dk_dp[rec] = interior ? v : NAN;
        if (out->dk_dp_stderr) out->dk_dp_stderr[rec] = interior ? e : NAN;
      }
      double vs, es;
      reduce(ns, &vs, &es);
      if (out->dk_dscale) out->dk_dscale[g] = (b->run.kind_mfp == PTG_MFP_PER_MODE ? vs : 0.0) + dks_an[g];
      if (out->dk_dscale_stderr) out->dk_dscale_stderr[g] = b->run.kind_mfp == PTG_MFP_PER_MODE ? es : 0.0;
    }
    out->flights = fwd_flights + st[0];
    out->replayed = nlist;
    out->mismatched = st[11];
    out->kernel_ms = (double)fwd_ms + (double)rep_ms;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

extern "C" void ptg_batch_destroy(ptg_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  delete b;
}
