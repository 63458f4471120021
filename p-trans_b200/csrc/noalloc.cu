/*
 * noalloc.cu - ptg_transmission_noalloc: the gray-MFP transmission function
 * of ptg_transmission (persistent FP32 kernel) with no device or host memory
 * allocated by the call.
 *
 * Some hosts cannot allocate device memory once they are running: a Fortran
 * or MPI code whose device memory is reserved up front by another framework
 * (a fixed budget carved out at start-up), or a long-running service that
 * must not grow or fragment its footprint between requests.  For them the
 * kernel's scratch memory (work-queue counter, statistics, per-task tallies,
 * task and chunk tables, the tail-phase list) lives in one fixed static
 * device array, g_noalloc_scratch, sized for PTG_NOALLOC_MAX_TASKS tasks,
 * PTG_NOALLOC_MAX_CHUNKS work chunks and kMaxTail handed-over phonons (a
 * phonon past that capacity stays in the drain phase).  Every GPU that loads the library holds
 * the array until the process exits.
 *
 * Rules of use:
 *  - the first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture;
 *  - all calls share the array and it keeps the last call's contents; each
 *    call clears the parts that must start at zero.  Two calls whose GPU work
 *    overlaps (different host threads, or different handles on the same
 *    device) race on the array: serialise them.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "ptg_internal.h"

namespace {

constexpr int64_t kMaxTasks = PTG_NOALLOC_MAX_TASKS;
constexpr int64_t kMaxChunks = PTG_NOALLOC_MAX_CHUNKS;
constexpr int kMaxAngles = 64;
constexpr int kMaxTail = 65536;   /* tail-list phonons, kTailUnits float4 each */

/* layout of the scratch array, byte offsets (all 256-byte aligned) */
constexpr size_t kOffStats = 0;                                /* u64[kStatSlots] */
static_assert(ptg::kStatSlots * 8 <= 256, "stats region");
constexpr size_t kOffQueue = 256;                              /* int[8]        */
constexpr size_t kOffCounts = 512;                             /* u64[tasks]    */
constexpr size_t kOffLost = kOffCounts + 8 * kMaxTasks;        /* u64[tasks]    */
constexpr size_t kOffTasks = kOffLost + 8 * kMaxTasks;         /* float4[tasks] */
constexpr size_t kOffOmega = kOffTasks + 16 * kMaxTasks;       /* double[tasks] */
constexpr size_t kOffChunks = kOffOmega + 8 * kMaxTasks;       /* int4[chunks]  */
constexpr size_t kOffTail = kOffChunks + 16 * kMaxChunks;     /* float4[kTailUnits * tail] */
constexpr size_t kOffOrder = kOffTail + 16 * (size_t)ptg::kTailUnits * (size_t)kMaxTail; /* int[tail] */
constexpr size_t kScratchBytes = kOffOrder + 4 * ((size_t)kMaxTail + ptg::kTailOrderExtra);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct AngleTable {
  float cth[kMaxAngles];
  float sth[kMaxAngles];
};

/* Task table (lambda, cos, sin, omega / max omega) and chunk table
   (task, first local particle, count) for one gray run. */
__global__ void k_noalloc_tables(unsigned char* base, int64_t nmode, int64_t ntask,
                                 int64_t chunks_per_task, int64_t chunk_size, int64_t np_local,
                                 float lam, double max_omega, AngleTable ang) {
  float4* tasks = reinterpret_cast<float4*>(base + kOffTasks);
  const double* omega = reinterpret_cast<const double*>(base + kOffOmega);
  int4* chunks = reinterpret_cast<int4*>(base + kOffChunks);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask; t += stride) {
    const int64_t m = t % nmode, ia = t / nmode;
    tasks[t] = make_float4(lam, ang.cth[ia], ang.sth[ia], (float)(omega[m] / max_omega));
    for (int64_t c = 0; c < chunks_per_task; ++c) {
      const int64_t j0 = c * chunk_size;
      const int64_t cnt = (np_local - j0 < chunk_size) ? np_local - j0 : chunk_size;
      chunks[t * chunks_per_task + c] = make_int4((int)t, (int)j0, (int)cnt, 0);
    }
  }
}

std::mutex g_setup_mutex;
void* g_scratch_ptr[128] = {nullptr};

/* Device address of the scratch array on the current device (set-up once per
   device, with that device current). */
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= 128) return PTG_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PTG_ERR_CUDA;
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
  return PTG_OK;
}

}  // namespace

extern "C" int ptg_transmission_noalloc(ptg_handle* h, double mfp_nm, int32_t nangle, int64_t np,
                                        int32_t rank, int32_t nranks, uint64_t seed,
                                        double* transmit) {
  if (!h || !transmit) return PTG_ERR_INVALID;
  if (nangle < 2 || nangle > kMaxAngles || np < 1 || nranks < 1 || rank < 0 || rank >= nranks ||
      !(mfp_nm > 0.0))
    return PTG_ERR_INVALID;
  ptg::NoallocView v;
  if (ptg::handle_noalloc_view(h, &v) != PTG_OK) return PTG_ERR_INVALID;
  const int64_t nmode = (int64_t)v.spec->nb * v.spec->nk;
  const int64_t ntask = nmode * (nangle - 1);
  /* sizes beyond the fixed scratch are refused before any GPU work */
  if (ntask > kMaxTasks || nmode > kMaxTasks) return PTG_ERR_INVALID;
  const int64_t np_local = np > rank ? (np - rank + nranks - 1) / nranks : 0;
  if (np_local > 2147483647LL) return PTG_ERR_INVALID;
  int64_t chunk = v.opt.chunk > 0 ? v.opt.chunk : 64;
  int64_t per_task = np_local > 0 ? (np_local + chunk - 1) / chunk : 0;
  if (ntask * per_task > kMaxChunks) {
    per_task = kMaxChunks / (ntask > 0 ? ntask : 1);
    if (per_task < 1) return PTG_ERR_INVALID;
    chunk = (np_local + per_task - 1) / per_task;
    per_task = (np_local + chunk - 1) / chunk;
  }
  if (cudaSetDevice(v.device) != cudaSuccess) return PTG_ERR_CUDA;
  unsigned char* base = nullptr;
  int st = scratch_address(v.device, &base);
  if (st != PTG_OK) return st;
  cudaStream_t s = v.stream;
  AngleTable ang;
  memset(&ang, 0, sizeof(ang));
  const double half_pi = 3.14159265358979323846 * 0.5;
  for (int ia = 0; ia < nangle - 1; ++ia) {
    const double theta = 0.0 + (double)ia / (double)(nangle - 1) * half_pi;
    ang.cth[ia] = (float)cos(theta);
    ang.sth[ia] = (float)sin(theta);
  }
  const float lam = (mfp_nm == 1.0e10) ? INFINITY : (float)mfp_nm;
  unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + kOffStats);
  int* queue = reinterpret_cast<int*>(base + kOffQueue);
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(base + kOffCounts);
  unsigned long long* lost = reinterpret_cast<unsigned long long*>(base + kOffLost);
  /* clear what the kernel accumulates into; the tables are rewritten */
  if (cudaMemsetAsync(stats, 0, ptg::kStatSlots * sizeof(unsigned long long), s) != cudaSuccess ||
      cudaMemsetAsync(stats + 5, 0xFF, 2 * sizeof(unsigned long long), s) != cudaSuccess ||
      cudaMemsetAsync(queue, 0, 8 * sizeof(int), s) != cudaSuccess ||
      cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * ntask, s) != cudaSuccess ||
      cudaMemsetAsync(lost, 0, sizeof(unsigned long long) * ntask, s) != cudaSuccess ||
      cudaMemcpyAsync(base + kOffOmega, v.spec->omega.data(), sizeof(double) * nmode,
                      cudaMemcpyHostToDevice, s) != cudaSuccess)
    return PTG_ERR_CUDA;
  k_noalloc_tables<<<(unsigned)((ntask + 255) / 256 > 0 ? (ntask + 255) / 256 : 1), 256, 0, s>>>(
      base, nmode, ntask, per_task, chunk, np_local, lam, v.spec->max_omega, ang);
  if (cudaGetLastError() != cudaSuccess) return PTG_ERR_CUDA;
  ptg::RunF32 r;
  memset(&r, 0, sizeof(r));
  r.task = reinterpret_cast<const float4*>(base + kOffTasks);
  r.chunk = reinterpret_cast<const int4*>(base + kOffChunks);
  r.nchunk = (int32_t)(ntask * per_task);
  r.np = np;
  r.rank = rank;
  r.nranks = nranks;
  r.k0 = (uint32_t)seed;
  r.k1 = (uint32_t)(seed >> 32);
  r.c1 = 0;
  const int64_t maxf = v.opt.max_flights > 0 ? v.opt.max_flights : 10000000LL;
  r.max_flights = (uint32_t)(maxf < 4294967295LL ? maxf : 4294967295LL);
  r.ref_quirks = v.opt.ref_quirks;
  const int rt = v.opt.regen_threshold > 0 ? v.opt.regen_threshold : ptg::kDefaultRegen;
  r.regen_threshold = rt > 32 ? 32 : rt;
  r.fast_steps = (v.opt.tune_flags & 1) ? 0 : (v.opt.fast_steps > 0 ? v.opt.fast_steps : ptg::default_fast_steps(v.g32));
  const double lmin = fmin(v.geom->box[0], fmin(v.geom->box[1], v.geom->box[2]));
  r.fast_lambda_max = (float)(0.1 * lmin);
  r.counts = counts;
  r.lost = lost;
  r.stats = stats;
  r.queue = queue;
  /* the tail phase as in ptg_transmission (tune_flags bit 1 turns it off) */
  r.coop_lanes = (v.opt.tune_flags & 2) ? 0 : (v.opt.coop_lanes > 0 ? std::min(v.opt.coop_lanes, 32) : 32);
  r.stage_test = (v.opt.tune_flags & 4) ? 1 : 0;
  /* the block size rule of ptg_transmission: opt.block_size when it is a
     multiple of 32 up to 256, else 256 */
  const int bs = v.opt.block_size;
  const int block = (bs >= 32 && bs <= 256 && bs % 32 == 0) ? bs : 256;
  const size_t smem = ptg::dynamic_smem_bytes(v.g32, v.blob_bytes);
  int bps = 0;
  if (ptg::persistent_occupancy(block, smem, &bps, ptg::MODE_FORWARD, v.g32.has_ext != 0, v.g32.stage_smem != 0) !=
      cudaSuccess)
    return PTG_ERR_CUDA;
  if (v.opt.blocks_per_sm > 0 && v.opt.blocks_per_sm < bps) bps = v.opt.blocks_per_sm;
  if (bps < 1) bps = 1;
  const int grid = v.num_sms * bps;
  int tgrid = 0;
  if (r.coop_lanes > 0) {
    /* the drain kernel admits at most tail_cap hand-overs in total (one
       counter of all requests), so a grid with more lanes than the list
       holds keeps the extra phonons in the drain phase */
    r.tail = reinterpret_cast<float4*>(base + kOffTail);
    r.tail_cap = std::min(kMaxTail, grid * block);
    r.tail_order = reinterpret_cast<int*>(base + kOffOrder);
    int tbps = 0;
    if (ptg::tail_occupancy(block, smem, &tbps, ptg::MODE_FORWARD, v.g32.has_ext != 0, v.g32.stage_smem != 0) != cudaSuccess)
      return PTG_ERR_CUDA;
    tgrid = v.num_sms * (tbps < 1 ? 1 : tbps);
  }
  if (r.nchunk > 0) {
    if (ptg::launch_persistent_fp32(v.g32, r, grid, block, smem, s) != cudaSuccess)
      return PTG_ERR_CUDA;
    if (tgrid > 0 && (ptg::launch_tail_order(r, v.g32.box[0], s) != cudaSuccess ||
                      ptg::launch_tail_fp32(v.g32, r, tgrid, block, smem, s) != cudaSuccess))
      return PTG_ERR_CUDA;
  }
  /* the counts land in the caller's transmit array (ntask <= its length),
     then become count / np in place; the last angle is zero.  Statistics and
     queue counters come back into stack arrays. */
  int qerr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long sv[ptg::kStatSlots];
  if (cudaMemcpyAsync(transmit, counts, sizeof(unsigned long long) * ntask, cudaMemcpyDeviceToHost,
                      s) != cudaSuccess ||
      cudaMemcpyAsync(qerr, queue, sizeof(qerr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(sv, stats, sizeof(sv), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    for (int64_t t = 0; t < nmode * nangle; ++t) transmit[t] = 0.0;
    return PTG_ERR_CUDA;
  }
  /* the handle's record of its last call, as ptg_transmission leaves it
     (no kernel times: this entry records no events) */
  ptg_stats* L = v.last;
  memset(L, 0, sizeof(*L));
  L->flights = sv[0];
  L->lost = sv[1];
  L->capped = sv[2];
  L->samples = sv[3];
  L->max_traj_flights = sv[4];
  L->full_flights = sv[8];
  L->safe_balls = sv[9];
  L->coop_rounds = sv[12];
  L->coop_flights = sv[13];
  L->box_tests = sv[14];
  L->surface_tests = sv[15];
  L->launches = 1 + (r.nchunk > 0 ? (tgrid > 0 ? 4 : 1) : 0);
  L->grid = grid;
  L->block = block;
  L->h2d_bytes = sizeof(double) * nmode;
  L->d2h_bytes = sizeof(unsigned long long) * ntask + sizeof(qerr) + sizeof(sv);
  if (tgrid > 0) {
    ptg::tail_counts(qerr, r.tail_cap, &L->tail_phonons, &L->tail_refused);
    L->tail_flights = sv[17] >= sv[16] ? sv[17] - sv[16] : 0;
  }
  if (qerr[1] != 0) {
    /* a staging wait ran out: the counts are incomplete, return none */
    for (int64_t t = 0; t < nmode * nangle; ++t) transmit[t] = 0.0;
    return PTG_ERR_TIMEOUT;
  }
  for (int64_t t = 0; t < ntask; ++t) {
    unsigned long long c;
    memcpy(&c, &transmit[t], sizeof(c));
    transmit[t] = (double)c / (double)np;
  }
  for (int64_t t = ntask; t < nmode * nangle; ++t) transmit[t] = 0.0;
  /* the lost-phonon limit of ptg_transmission */
  if (v.opt.lost_limit > 0.0 && L->samples > 0 &&
      (double)L->lost > v.opt.lost_limit * (double)L->samples)
    return PTG_ERR_LOST;
  return PTG_OK;
}
