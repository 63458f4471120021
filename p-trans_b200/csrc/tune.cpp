/*
 * tune.cpp - ptg_autotune: picks the persistent kernel's launch and
 * scheduling parameters for one geometry, spectrum and run.
 *
 * No counterpart in the reference (its OpenMP loop has a fixed static
 * schedule, src/RTMCphon.f90:1573).  Coordinate descent: starting from the
 * handle's options, each parameter in turn takes every value of its
 * candidate list while the others stay fixed, and keeps the value with the
 * smallest transport-kernel time (best of `reps` calls of ptg_kappa with the
 * caller's run in FP32).  A change is kept only when it gains more than 1%,
 * so timing noise does not move the result.  Every trial computes the same
 * trajectories (they depend only on their Philox counters), so the tuner
 * changes speed, never results.
 *
 * Parameters and candidates:
 *   bvh_leaf        1 2 4 8 16    (only when some grain has a BVH)
 *   block_size      128 256
 *   blocks_per_sm   1 2
 *   coop_lanes      4 8 16 32
 *   fast_steps      4 8 16
 *   regen_threshold 1 2 4 8
 *   chunk           32 64 128
 */
#include <cstring>
#include <vector>

#include "ptg_internal.h"

namespace {

struct Param {
  int32_t ptg_options::*i32;
  int64_t ptg_options::*i64;
  std::vector<long long> values;
};

int time_once(ptg_handle* h, const ptg_run* run, int reps, double* ms) {
  ptg_run r = *run;
  r.precision = PTG_PREC_FP32;
  double best = 1e300;
  for (int i = 0; i < reps; ++i) {
    ptg_kappa_out out;
    memset(&out, 0, sizeof(out));
    int st = ptg_kappa(h, &r, &out);
    if (st != PTG_OK && st != PTG_ERR_LOST) return st;
    ptg_stats s;
    st = ptg_last_stats(h, &s);
    if (st != PTG_OK) return st;
    if (s.kernel_ms < best) best = s.kernel_ms;
  }
  *ms = best;
  return PTG_OK;
}

}  // namespace

extern "C" int ptg_autotune(ptg_handle* h, const ptg_run* run, int32_t reps, ptg_options* best,
                            double* best_ms) {
  try {
    if (!h || !run || !best) return PTG_ERR_INVALID;
    if (reps < 1) reps = 1;
    ptg_options cur;
    int st = ptg_get_options(h, &cur);
    if (st != PTG_OK) return st;
    const ptg_options start = cur;
    const bool has_bvh = ptg::handle_has_bvh(h);
    std::vector<Param> params;
    if (has_bvh) params.push_back({&ptg_options::bvh_leaf, nullptr, {1, 2, 4, 8, 16}});
    params.push_back({&ptg_options::block_size, nullptr, {128, 256}});
    params.push_back({&ptg_options::blocks_per_sm, nullptr, {1, 2}});
    params.push_back({&ptg_options::coop_lanes, nullptr, {4, 8, 16, 32}});
    params.push_back({&ptg_options::fast_steps, nullptr, {4, 8, 16}});
    params.push_back({&ptg_options::regen_threshold, nullptr, {1, 2, 4, 8}});
    params.push_back({nullptr, &ptg_options::chunk, {32, 64, 128}});
  
    double cur_ms = 0.0;
    st = time_once(h, run, reps, &cur_ms);
    if (st != PTG_OK) { ptg_set_options(h, &start); return st; }
    for (const Param& p : params) {
      ptg_options keep = cur;
      double keep_ms = cur_ms;
      for (long long v : p.values) {
        ptg_options trial = cur;
        if (p.i32) {
          if (trial.*(p.i32) == (int32_t)v) continue;
          trial.*(p.i32) = (int32_t)v;
        } else {
          if (trial.*(p.i64) == (int64_t)v) continue;
          trial.*(p.i64) = (int64_t)v;
        }
        st = ptg_set_options(h, &trial);
        if (st != PTG_OK) { ptg_set_options(h, &start); return st; }
        double ms = 0.0;
        st = time_once(h, run, reps, &ms);
        if (st != PTG_OK) { ptg_set_options(h, &start); return st; }
        if (ms < keep_ms * 0.99) { keep = trial; keep_ms = ms; }
      }
      cur = keep;
      cur_ms = keep_ms;
      st = ptg_set_options(h, &cur);
      if (st != PTG_OK) { ptg_set_options(h, &start); return st; }
    }
    *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}
