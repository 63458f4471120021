/*
 * ptg_internal.h - host-side types shared by the C ABI implementation and the
 * kernel launchers of the B200 RTMC phonon transport library.
 */
#ifndef PTG_INTERNAL_H
#define PTG_INTERNAL_H

#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/ptrans_gpu.h"

#include <nvtx3/nvToolsExt.h>
#include <new>

namespace ptg {

/* Allocation-failure injection (ptg_debug_fail_allocations): true when the
   allocation about to be made must fail; alloc_check() throws
   std::bad_alloc then. */
bool alloc_should_fail();
void alloc_check();

/* An NVTX range over a scope: the host-side phases of each entry point
   (transport launches, reductions, adjoint passes) show by name in Nsight
   Systems and in ncu --nvtx filters; without a tool attached it costs a
   call that returns at once. */
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};


/* Owning, structure-of-arrays copy of a built geometry (ptg_geometry). */
struct GeomSoA {
  double box[3] = {0, 0, 0};
  double scope[2] = {1, 1};
  int32_t face_kind[6] = {0, 0, 0, 0, 0, 0};
  int32_t kind_grain = PTG_GRAIN_VORONOI, ngrain = 0, igrain_fill = -1, nmaterial = 1;
  std::vector<int32_t> grain_begin, grain_incident;
  std::vector<double> grain_generatrix;
  std::vector<int32_t> shape, nvertex, vertex_begin, kind_trans, grain_inside, grain_outside,
      internal, incident, material1, material2;
  std::vector<double> vertex, normal, tangent, center, radius, specularity, trans_param;
  ptg_geometry view;  /* points into the vectors above */

  int32_t nsurf() const { return (int32_t)shape.size(); }
  int32_t ngrain_total() const { return (int32_t)grain_incident.size(); }
  void make_view();
};

/* Copies a caller-provided ptg_geometry after validating it. */
int copy_geometry(const ptg_geometry* g, GeomSoA* out, std::string* why);
/* Builds from the raw model (src/RTMCphon.f90:894-1491). */
int build_geometry(const ptg_model* m, GeomSoA* out, std::string* why);

/* Spectrum copy with the derived per-mode quantities. */
struct SpecSoA {
  int32_t nb = 0, nk = 0;
  double rtemp = 300, vol = 1, max_omega = 1;
  std::vector<double> omega, tau, vel, mfp, weight;
  int nmode() const { return nb * nk; }
};
int copy_spectrum(const ptg_spectrum* s, SpecSoA* out, std::string* why);

/* Per-task description shared by the launchers. */
struct TaskHost {
  double lambda;  /* nm; 1e10 ballistic; <= 0 not simulated */
  double cth, sth;
  double omega;
};

/* Numbering helpers for ptg_run (include/ptrans_gpu.h). */
int64_t run_ntask(const SpecSoA& s, const ptg_run* r);
bool run_valid(const SpecSoA& s, const ptg_run* r, std::string* why);
void run_tasks(const SpecSoA& s, const ptg_run* r, std::vector<TaskHost>* tasks);

/* Host FP64 kappa assembly (effectiveMFP + fileoutput kappa sum). */
struct ModeConst {
  std::vector<double> K;      /* C*w*v/(3*vol*nqfbz): kappa per unit EMFP [m] */
  std::vector<double> W;      /* C*w*v: flux weight of the per-bin averages    */
  std::vector<double> mfp_m;  /* bulk MFP [m] after the tau rescale            */
  std::vector<int32_t> bin;   /* frequency bin or -1                           */
};
void mode_constants(const SpecSoA& s, const ptg_run* r, ModeConst* mc);
void simpson_weights(int nangle, double box_x, std::vector<double>* coef, double* dS);

}  // namespace ptg

#include "kernels.h"

namespace ptg {

/* What ptg_transmission_noalloc reads from a handle (no copies made). */
struct NoallocView {
  GeoF32 g32;
  size_t blob_bytes;
  int device, num_sms;
  cudaStream_t stream;
  ptg_options opt;
  const SpecSoA* spec;
  const GeomSoA* geom;
  ptg_stats* last;   /* the handle's record of its last call (plain struct) */
};
int handle_noalloc_view(ptg_handle* h, NoallocView* v);

/* Phonons handed to the tail list and hand-overs refused for lack of room,
   from the drain kernel's queue counters (queue[2] long, queue[4] short,
   queue[5] all requests) and the list's capacity. */
inline void tail_counts(const int* queue, int cap, uint64_t* handed, uint64_t* refused) {
  const int64_t lng = queue[2] < 0 ? 0 : queue[2], sht = queue[4] < 0 ? 0 : queue[4];
  int64_t got = lng + sht;
  if (got > cap) got = cap;
  const int64_t req = queue[5] < 0 ? 0 : queue[5];
  *handed = (uint64_t)got;
  *refused = (uint64_t)(req > got ? req - got : 0);
}

/* FP32 geometry blob (host copy) of a built geometry; grains with more than
   kBvhMinCand candidates get a BVH with leaves of bvh_leaf surfaces
   (bvh_leaf < 0: none, linear candidate scans everywhere). */
constexpr int kBvhMinCand = 32;
constexpr int kBvhDefaultLeaf = 4;
int blob_from_geometry(const GeomSoA& G, int bvh_leaf, std::vector<float4>* out, BlobLayout* lay,
                       std::string* why);
/* Binned-SAH BVH over boxes lo/hi (3 floats each): nodes (2 float4 each,
   children and leaf ranges absolute: node_base, cand_base added) and the
   primitive order of the leaves.  Returns the node count. */
int bvh_build(const std::vector<float>& lo, const std::vector<float>& hi, int leaf, int max_depth,
              int cand_base, int node_base, std::vector<float4>* nodes, std::vector<int>* order);
/* True when some grain of the handle's geometry has more than kBvhMinCand
   candidate surfaces (a BVH unless bvh_leaf < 0). */
bool handle_has_bvh(const ptg_handle* h);
/* Host FP64 kappa assembly (see api.cpp). */
int assemble_host(const SpecSoA& S, const ptg_run* run, double box_x, const uint64_t* counts,
                  ptg_kappa_out* out, std::vector<double>* wtask, double* dk_ds_an);

}  // namespace ptg

#endif
