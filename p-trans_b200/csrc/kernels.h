/*
 * kernels.h - device data layouts and host-callable launchers of the
 * transport and reduction kernels.
 */
#ifndef PTG_KERNELS_H
#define PTG_KERNELS_H

#include <cuda_runtime.h>
#include <stdint.h>

namespace ptg {

/* ---------------- plain FP64 kernel ------------------------------------- */

/* Built geometry in device memory, FP64 structure of arrays (the
   ptg_geometry fields the transport reads). */
struct Geo64 {
  const double* vertex;      /* closed polygons, 3 per vertex        */
  const double* normal;      /* 3 per surface                        */
  const double* tangent;     /* 9 per surface, column-major          */
  const double* center;      /* 3 per surface                        */
  const double* radius;
  const double* spec;
  const double* tparam;
  const int* shape;
  const int* nvertex;
  const int* vbegin;
  const int* kind_trans;
  const int* gout;
  const int* internal;
  const int* incident;
  const int* grain_begin;
  const int* grain_incident;
  const double* grain_gen;   /* 3 per grain                          */
  double box[3];
  double scope[2];
  int face_kind[6];
  int kind_grain, ngrain, igrain_fill, nmaterial;
  double max_omega;
};

/* Per task: lambda [nm] (1e10 ballistic, <= 0 skipped), cos/sin of the
   incident angle, mode omega. */
struct Task64 {
  double lambda, cth, sth, omega;
};

struct Run64 {
  const Task64* task;
  int64_t ntask;
  int64_t np;                 /* particles per task (all ranks)          */
  int64_t np_local;           /* particles of this rank per task         */
  int32_t rank, nranks;
  uint32_t k0, k1, c1;        /* Philox key and stream word              */
  int64_t max_flights;
  int32_t ref_quirks;
  unsigned long long* counts; /* [ntask]                                 */
  unsigned long long* lost;   /* [ntask]                                 */
  unsigned long long* stats;  /* flights, lost, capped, samples          */
  /* replay of one task (replay_task >= 0) */
  int64_t replay_task;
  int* end_side;
  unsigned* flights;
  double* final_pos;
};

cudaError_t launch_plain_fp64(const Geo64& g, const Run64& r, cudaStream_t st, int* grid,
                              int* block);

/* ---------------- persistent FP32 kernel -------------------------------- */

/* Surface record types in the FP32 blob. */
/* REC_CAP: capped cylinder, its (unit axis, half length) in the edge array */
enum { REC_POLY = 1, REC_SPHERE = 2, REC_CYL = 3, REC_CAP = 4 };
enum { REC_INTERIOR = 1 << 8 };

/* Offsets (in 16-byte units) of the sections of the FP32 geometry blob. */
struct BlobLayout {
  int hot;          /* float4[2*nsurf]: A = shape data, B = int4 (type, e0, ne, geom) */
  int cold;         /* float4[3*nsurf]: (t1,spec) (t2,tparam) (n, kind|gout<<8)      */
  int edge;         /* float4[nedge]  : in-plane inward edge normal m, m.v           */
  int cand_begin;   /* int[ngrain_total+1]                                           */
  int cand;         /* int[ncand]                                                    */
  int start;        /* voronoi: float4 (generatrix, grain); bricks: int2 (surf, grain) */
  int bvh_root;     /* int[ngrain_total]: root node of the grain's BVH, -1 linear scan */
  int bvh_node;     /* float4[2*nnode]: (lo, a) (hi, b), see bvh.cpp                  */
  int nbvh;         /* BVH nodes in the blob (0: every grain scans linearly)          */
  int ncap;         /* capped-cylinder records in the blob                            */
  int total;        /* blob size in 16-byte units                                    */
  int nstart;
};

struct GeoF32 {
  const float4* blob;  /* device blob (global memory)                    */
  BlobLayout lay;
  float box[3];
  float scope[2];
  float eps;           /* absolute geometric tolerance [nm]              */
  int periodic_mask;   /* bit f set: box face f is periodic              */
  int kind_grain, igrain_fill, nmaterial;
  int stage_smem;      /* 1: copy the blob to shared memory (bulk copy)  */
  int node_stage;      /* else: float4 units of the BVH node region (its  */
                       /*    top levels, breadth first) copied instead    */
  int has_ext;         /* 1: a BVH or capped cylinders (kernels built for  */
                       /*    them; the others leave both out)             */
};

/* One geometry of a batched launch (device table, read through the cache). */
struct GeoEntry {
  const float4* blob;
  BlobLayout lay;
  float box[3];
  float scope[2];
  float eps;
  float fast_lambda_max;
  int periodic_mask, kind_grain, igrain_fill, nmaterial;
  long long np;                /* particles per task of this geometry        */
  unsigned k0, k1, c1;         /* Philox key and stream word                 */
  int task_base;               /* first global task of this geometry         */
  int nsurf;                   /* its surfaces (adjoint replay)               */
  int adj_base;                /* its adjoint accumulators' first element    */
};

/* Per task (FP32): lambda (inf = ballistic, <= 0 skipped), cos, sin, omega/max_omega */
struct RunF32 {
  const float4* task;
  const int4* chunk;          /* (task, first local particle, count, 0) in LPT order */
  int32_t nchunk;
  int64_t np;
  int32_t rank, nranks;
  uint32_t k0, k1, c1;
  uint32_t max_flights;
  int32_t ref_quirks;
  int32_t regen_threshold;
  int32_t fast_steps;         /* max safe-distance p-p flights per iteration (0: off) */
  float fast_lambda_max;      /* tasks with a smaller MFP use the fast path           */
  int32_t coop_lanes;         /* once the queue is dry, a warp with at most this many
                                 live phonons moves them to the tail list, where
                                 each gets a warp of its own that advances it 32
                                 flights a round (0: off)                         */
  float4* tail;               /* tail list: kTailUnits float4 per phonon           */
  int32_t tail_cap;           /* its capacity in phonons                           */
  int32_t* tail_order;        /* the tail phase takes list slots in this order
                                 (launch_tail_order), else front then back         */
  int32_t stage_test;         /* test only: set up the shared-memory staging
                                 barrier without issuing the copy, so its
                                 bounded wait runs out (PTG_ERR_TIMEOUT)          */
  unsigned long long* counts;
  unsigned long long* lost;
  /* flights, lost, capped, samples, max trajectory flights,
     t_start (min), t_drain (min), t_end (max) in globaltimer ns,
     flights taken with the intersection test, safe balls built */
  unsigned long long* stats;
  int* queue;                 /* [0] next chunk, [1] error flags, [2] / [4] phonons
                                 put at the front / back of the tail list, [3]
                                 next tail-list phonon, [5] tail-list requests
                                 (8 ints) */
  /* adjoint support */
  unsigned long long* tlist;  /* mode 1: sample ids of transmitted phonons         */
  unsigned long long tlist_cap;
  const unsigned long long* alist;  /* mode 2: sample ids to replay               */
  long long alist_n;
  const float* wsample;       /* mode 2: d kappa / d T_task / np, per task         */
  double* adj;                /* mode 2: [kAdjBatches][nsurf + 1] accumulators     */
  int nsurf;
  /* mode 3: per replayed sample, positions (3 floats) at trace_off[t] ..
     trace_off[t+1] (trace NULL: counting pass), position count and exit */
  float* trace;
  const long long* trace_off;
  long long* trace_npos;
  int* trace_end;
  /* batched launch: geometry table and the geometry of every global task */
  const GeoEntry* geos;
  const int* task_geo;
};

/* u64 statistics slots of a transport launch: 0 flights, 1 lost, 2 capped,
   3 samples, 4 longest trajectory, 5-7 globaltimer start / queue dry / end,
   8 full-test flights, 9 safe balls, 10 listed samples, 11 replay
   mismatches, 12 cooperative rounds, 13 cooperative flights, 14 BVH boxes,
   15 surfaces tested, 16 flights of phonons handed to the tail phase before
   the hand-over, 17 flights of phonons that ended in the tail phase. */
constexpr int kStatSlots = 24;

/* Scheduling defaults of the persistent kernel (ptg_options 0 = these):
   idle lanes before a warp refills, fast-path flights per lane and
   iteration (structures whose grains are scanned linearly take short
   fast-path bursts, their full flights being cheap: thin film 16.5 ->
   15.8 ms, Voronoi 312 -> 305 ms at 4 against 8; those with a BVH or capped
   cylinders amortise dearer full flights over longer ones: C3 766 / 740 /
   733 ms and C4 3877 -> 3817 ms at 4 / 8 / 12, and with three drain blocks
   per SM C4 3661 -> 3592 ms at 12 -> 20; the batched launch keeps 8). */
constexpr int kDefaultRegen = 2;
constexpr int kDefaultFastSteps = 8;
constexpr int kDefaultFastStepsPlain = 4;
constexpr int kDefaultFastStepsExt = 20;
inline int default_fast_steps(const GeoF32& g) {
  return g.has_ext ? kDefaultFastStepsExt : kDefaultFastStepsPlain;
}

/* Replays are split in this many interleaved batches (sample % kAdjBatches)
   whose spread gives the standard error of the adjoint estimates. */
constexpr int kAdjBatches = 8;
/* kernel modes: forward, forward + list of transmitted samples, adjoint replay */
/* forward tallies; + list of transmitted samples; adjoint replay of a list;
   trace replay of a list (one-lane full flights, positions recorded) */
enum { MODE_FORWARD = 0, MODE_LIST = 1, MODE_ADJOINT = 2, MODE_TRACE = 3 };

cudaError_t launch_persistent_fp32(const GeoF32& g, const RunF32& r, int grid, int block,
                                   size_t smem, cudaStream_t st, int mode = MODE_FORWARD);
/* The tail phase after it (forward, list and adjoint modes): the phonons
   the drain phase left in r.tail, one per warp. */
/* Orders the tail list for the tail phase (r.tail_order: tail_cap ints and
   kTailOrderExtra more for a histogram and cursors): longest expected
   remaining walk first.  A memset and two kernels between the drain and the
   tail launch on the same stream; x_len is the box length along x. */
constexpr int kTailOrderExtra = 256;
cudaError_t launch_tail_order(const RunF32& r, float x_len, cudaStream_t st);
cudaError_t launch_tail_fp32(const GeoF32& g, const RunF32& r, int grid, int block, size_t smem,
                             cudaStream_t st, int mode = MODE_FORWARD);
cudaError_t tail_occupancy(int block, size_t smem, int* blocks_per_sm, int mode = MODE_FORWARD,
                           bool bvh = false, bool whole = true);
/* Batched launch over several geometries (geometry in global memory):
   forward, list (ids of transmitted samples as (global task << 32) |
   particle) or adjoint replay of such a list. */
cudaError_t launch_persistent_batch(const RunF32& r, int grid, int block, cudaStream_t st,
                                    bool bvh, int mode = MODE_FORWARD);
cudaError_t persistent_batch_occupancy(int block, int* blocks_per_sm, bool bvh,
                                       int mode = MODE_FORWARD);
/* float4 per phonon in the tail list: the state of a phonon handed from the
   drain phase to the tail phase (position, direction, free path, MFP, the
   ball centre and radii, grain, last surface, task, omega, sample id,
   flight, adjoint terms, second ball). */
constexpr int kTailUnits = 7;
/* Shared memory for staged BVH nodes when the whole blob is not staged:
   64 KB, the top ten or so levels of the trees, small enough that two
   blocks of the tail kernel (28.5 KB of its own) still fit on an SM. */
constexpr int kNodeStageUnits = 4096;
/* Dynamic shared memory of a transport launch: the whole blob, or the
   staged BVH nodes, or none. */
inline size_t dynamic_smem_bytes(const GeoF32& g, size_t blob_bytes) {
  if (g.stage_smem) return blob_bytes;
  return (size_t)g.node_stage * 16u;
}
/* Fills the chunk table (task, first local particle, count, 0): per_task
   chunks of csz particles for each task of `order`, in that order. */
cudaError_t launch_expand_chunks(const int* order, int norder, int per_task, int csz, int np_local,
                                 int4* chunks, cudaStream_t st);
/* Violations recorded by the bounds-checked build (PT_CHECK); other builds
   return cudaErrorNotSupported. */
cudaError_t check_report(long long* count, int* code, int* index, bool reset);
/* Residency of the persistent kernel for a block size and shared memory. */
cudaError_t persistent_occupancy(int block, size_t smem, int* blocks_per_sm,
                                 int mode = MODE_FORWARD, bool bvh = false, bool whole = true);

/* ---------------- FP64 kappa reduction ---------------------------------- */

struct ReduceIn {
  const unsigned long long* counts;  /* [ntask]                          */
  int64_t nmode;
  int32_t nangle, ns, kind_mfp, nbins;
  double np;                         /* particles per task                */
  double dS;                         /* Simpson step * 1.5 * Lx           */
  double tnorm;                      /* 0.75 * Lx                         */
  const double* coef;                /* [nangle] Simpson c_a sin cos      */
  const double* K;                   /* [nmode]                           */
  const double* W;                   /* [nmode]                           */
  const double* mfp_m;               /* [nmode] bulk MFP [m]              */
  const int* bin;                    /* [nmode]                           */
  const double* grid;                /* [ns] (GRID)                       */
  /* scratch and outputs */
  double* tc;                        /* [nmode] kappa per mode            */
  double* kv;                        /* [nmode] kappa variance per mode   */
  double* bw;                        /* [nmode] W * <T>                   */
  double* bv;                        /* [nmode] W^2 var<T>                */
  double* emfp_nm;                   /* [nmode]                           */
  double* transmit;                  /* [nmode*ns*nangle] or null         */
  double* result;                    /* [2 + 3*nbins]: kappa, var, (sumW, sumWT, sumW2V) per bin */
};

cudaError_t launch_kappa_reduce(const ReduceIn& in, cudaStream_t st);

/* Batched reduction: the same spectrum for ngeo geometries whose counts are
   stored one after another (ntask_per_geo each); per geometry np and box x.
   result: [ngeo][2 + 3*nbins]. */
struct ReduceBatchIn {
  ReduceIn base;               /* counts, coef, K, W, mfp_m, bin, grid, nbins... */
  int ngeo;
  long long ntask_per_geo;
  const double* np_geo;        /* [ngeo] */
  const double* dS_geo;        /* [ngeo] */
  const double* tnorm_geo;     /* [ngeo] */
};
cudaError_t launch_kappa_reduce_batch(const ReduceBatchIn& in, cudaStream_t st);

}  // namespace ptg

#endif
