/*
 * kernels_fp64.cu - the plain FP64 transport kernel: one phonon per thread,
 * the reference's linear scan of the box grain plus the current grain per
 * free flight, the reference's intersection / reflection / transmission
 * arithmetic in FP64, the 1e-7 nm nudge and the out-of-box check
 * (calcTransmit and helpers, src/RTMCphon.f90:1608-2414, 2883-3301).
 *
 * It is the comparator of the persistent FP32 kernel and the replay target of
 * the CPU oracle: this file is compiled with --fmad=false so every a*b+c is
 * rounded twice, exactly as the host restatement computes it.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp64_math.cuh"
#include "kernels.h"
#include "philox.cuh"

namespace ptg {

namespace {

constexpr double kSmall = 1.0e-5;       /* SMALL_VAL, src/RTMCphon.f90:67 */
constexpr double kBallistic = 1.0e10;   /* src/RTMCphon.f90:1686          */

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

struct Draw {
  Key2 key;
  uint32_t c1, slo, shi;
  __device__ void block(uint32_t flight, uint32_t sub, double* d0, double* d1) const {
    const uint4 p = philox10(flight, sub | c1, slo, shi, key);
    *d0 = u52d(p.x, p.y);
    *d1 = u52d(p.z, p.w);
  }
};

/* Convex-polygon sign test of src/RTMCphon.f90:2942-2955 / 2961-2983. */
__device__ bool in_polygon(const double* v, int n, const double* Rh) {
  double c1[3], ci[3], Ra[3], Rb[3];
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) {
      Ra[d] = v[3 * (i + 1) + d] - v[3 * i + d];
      Rb[d] = Rh[d] - v[3 * i + d];
    }
    cross3(Ra, Rb, ci);
    if (i == 0) {
      c1[0] = ci[0]; c1[1] = ci[1]; c1[2] = ci[2];
    } else if (dot3(c1, ci) < 0.0) {
      return false;
    }
  }
  return true;
}

/* Capped cylinder (extension): unit axis and half length from the axis end
   points A = vertex 0, B = vertex 1. */
__device__ void capped_axis(const Geo64& g, int k, double* a, double* hl) {
  const double* v = g.vertex + 3 * (size_t)g.vbegin[k];
  double e[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
  const double len = sqrt(dot3(e, e));
  for (int d = 0; d < 3; ++d) a[d] = e[d] / len;
  *hl = 0.5 * len;
}

/* Nearest strictly positive hit of the lateral surface (within the caps)
   and the two cap discs (within the radius). */
__device__ bool capped_distance(const Geo64& g, int k, const double* R0, const double* D,
                                double* L) {
  double a[3], hl;
  capped_axis(g, k, a, &hl);
  const double* C = g.center + 3 * k;
  double w[3] = {R0[0] - C[0], R0[1] - C[1], R0[2] - C[2]};
  const double s0 = dot3(w, a), ds = dot3(D, a);
  double wp[3], dp[3];
  for (int d = 0; d < 3; ++d) {
    wp[d] = w[d] - s0 * a[d];
    dp[d] = D[d] - ds * a[d];
  }
  const double r2 = g.radius[k] * g.radius[k];
  double best = 0.0;
  bool hit = false;
  const double A2 = dot3(dp, dp);
  if (A2 > 0.0) {
    const double B = dot3(wp, dp), Cc = dot3(wp, wp) - r2;
    const double disc = B * B - A2 * Cc;
    if (disc >= 0.0) {
      const double sq = sqrt(disc);
      const double t[2] = {(-B - sq) / A2, (-B + sq) / A2};
      for (int i = 0; i < 2; ++i) {
        if (!(t[i] > 0.0) || (hit && !(t[i] < best))) continue;
        if (fabs(s0 + t[i] * ds) <= hl) { best = t[i]; hit = true; }
      }
    }
  }
  if (ds != 0.0) {
    for (int i = 0; i < 2; ++i) {
      const double c = (i == 0) ? -hl : hl;
      const double t = (c - s0) / ds;
      if (!(t > 0.0) || (hit && !(t < best))) continue;
      double q[3];
      for (int d = 0; d < 3; ++d) q[d] = wp[d] + t * dp[d];
      if (dot3(q, q) <= r2) { best = t; hit = true; }
    }
  }
  if (!hit) return false;
  *L = best;
  return true;
}

/* Outward normal of the nearer piece: cap (+-axis) or mantle (radial). */
__device__ void capped_normal(const Geo64& g, int k, const double* R, double* N) {
  double a[3], hl;
  capped_axis(g, k, a, &hl);
  const double* C = g.center + 3 * k;
  double w[3] = {R[0] - C[0], R[1] - C[1], R[2] - C[2]};
  const double sa = dot3(w, a);
  double wp[3];
  for (int d = 0; d < 3; ++d) wp[d] = w[d] - sa * a[d];
  const double rho = sqrt(dot3(wp, wp));
  if (fabs(fabs(sa) - hl) < fabs(rho - g.radius[k])) {
    const double sg = (sa < 0.0) ? -1.0 : 1.0;
    for (int d = 0; d < 3; ++d) N[d] = sg * a[d];
  } else {
    for (int d = 0; d < 3; ++d) N[d] = wp[d] / rho;
  }
}

/* calcSurfaceDistance dispatch, src/RTMCphon.f90:2883-3088 */
__device__ bool surface_distance(const Geo64& g, int k, const double* R0, const double* D,
                                 double* L) {
  const int sh = g.shape[k];
  if (sh == 1) {
    const double* N = g.normal + 3 * k;
    const double cosangle = dot3(D, N);
    if (cosangle <= 0.0) return false;
    const double* v = g.vertex + 3 * (size_t)g.vbegin[k];
    double w[3] = {v[0] - R0[0], v[1] - R0[1], v[2] - R0[2]};
    const double Lh = dot3(w, N) / cosangle;
    if (Lh < 0.0) return false;
    double Rh[3];
    for (int d = 0; d < 3; ++d) Rh[d] = R0[d] + D[d] * Lh;
    if (!in_polygon(v, g.nvertex[k], Rh)) return false;
    *L = Lh;
    return true;
  }
  if (sh == 4) return capped_distance(g, k, R0, D, L);
  const double* C = g.center + 3 * k;
  const double r = g.radius[k];
  const double r2 = r * r;
  if (sh == 2) {
    double Rsc[3] = {C[0] - R0[0], C[1] - R0[1], C[2] - R0[2]};
    const double RD = dot3(Rsc, D);
    const double RR = dot3(Rsc, Rsc);
    if (RR > r2 - 1e-10) {
      if (RD <= 0.0) return false;
    }
    const double Dd = RD * RD + r2 - RR;
    if (Dd < 0.0) return false;
    const double sq = sqrt(Dd);
    const double L1 = RD - sq, L2 = RD + sq;
    if (L1 > 0.0) *L = L1;
    else if (L2 > 0.0) *L = L2;
    else return false;
    return true;
  }
  /* z-axis cylinder clipped to 0 <= z <= Lz */
  const double Rs0 = C[0] - R0[0], Rs1 = C[1] - R0[1];
  double t0 = D[0], t1 = D[1];
  const double nv = t0 * t0 + t1 * t1 + 0.0 * 0.0;
  const double snv = sqrt(nv);
  t0 = t0 / snv;
  t1 = t1 / snv;
  const double RD = Rs0 * t0 + Rs1 * t1;
  const double RR = Rs0 * Rs0 + Rs1 * Rs1;
  const double Dd = RD * RD + r2 - RR;
  if (Dd < 0.0) return false;
  const double sq = sqrt(Dd);
  const double L1 = RD - sq, L2 = RD + sq;
  double Lh;
  if (L1 > 0.0) Lh = L1;
  else if (L2 > 0.0) Lh = L2;
  else return false;
  Lh = Lh / sqrt(D[0] * D[0] + D[1] * D[1]);
  const double z = R0[2] + D[2] * Lh;
  if (z < 0.0 || g.box[2] < z) return false;
  *L = Lh;
  return true;
}

/* calcSurfaceNormal*, src/RTMCphon.f90:3119-3179 */
__device__ void surface_normal(const Geo64& g, int k, const double* R, double* N) {
  const int sh = g.shape[k];
  if (sh == 1) {
    N[0] = g.normal[3 * k]; N[1] = g.normal[3 * k + 1]; N[2] = g.normal[3 * k + 2];
    return;
  }
  if (sh == 4) {
    capped_normal(g, k, R, N);
    return;
  }
  const double* C = g.center + 3 * k;
  double Rcs[3];
  if (sh == 2) {
    Rcs[0] = R[0] - C[0]; Rcs[1] = R[1] - C[1]; Rcs[2] = R[2] - C[2];
  } else {
    Rcs[2] = 0.0; Rcs[0] = R[0] - C[0]; Rcs[1] = R[1] - C[1];
  }
  const double rr = dot3(Rcs, Rcs);
  const double inv = 1.0 / sqrt(rr);
  for (int d = 0; d < 3; ++d) N[d] = Rcs[d] * inv;
  if (rr > g.radius[k] * g.radius[k])
    for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
}

/* calcSurfaceRotation*, src/RTMCphon.f90:3181-3301 (column-major) */
__device__ void surface_rotation(const Geo64& g, int k, const double* R, double* Rm) {
  const int sh = g.shape[k];
  if (sh == 1) {
    for (int d = 0; d < 9; ++d) Rm[d] = g.tangent[9 * k + d];
    return;
  }
  const double* C = g.center + 3 * k;
  double n[3];
  if (sh == 4) {
    capped_normal(g, k, R, n);
  } else if (sh == 2) {
    double Rcs[3] = {R[0] - C[0], R[1] - C[1], R[2] - C[2]};
    const double inv = 1.0 / sqrt(dot3(Rcs, Rcs));
    for (int d = 0; d < 3; ++d) n[d] = Rcs[d] * inv;
  } else {
    double Nn[3] = {R[0] - C[0], R[1] - C[1], 0.0};
    const double inv = 1.0 / sqrt(dot3(Nn, Nn));
    for (int d = 0; d < 3; ++d) n[d] = Nn[d] * inv;
  }
  Rm[6] = n[0]; Rm[7] = n[1]; Rm[8] = n[2];
  const double pole = (sh == 3) ? fabs(n[0]) : fabs(n[2]);
  if (pole == 1.0 || (n[0] * n[0] == 0.0 && n[1] * n[1] == 0.0)) {
    Rm[3] = 0; Rm[4] = 1; Rm[5] = 0; Rm[0] = 1; Rm[1] = 0; Rm[2] = 0;
  } else {
    const double q = sqrt(n[0] * n[0] + n[1] * n[1]);
    Rm[3] = -n[1] / q; Rm[4] = n[0] / q; Rm[5] = 0.0;
    cross3(&Rm[3], &Rm[6], &Rm[0]);
  }
}

/* determinTransmit threshold, src/RTMCphon.f90:2384-2413 */
__device__ double threshold(const Geo64& g, int k, double omega, double od) {
  const int kt = g.kind_trans[k];
  const double tp = g.tparam[k];
  if (kt == 1) return tp;
  if (kt == 2 || kt == 3) {
    if (g.nmaterial == 1) return 1.0 / (tp * omega / g.max_omega + 1.0);
    const double t11 = 1.0 / (tp + 1.0);
    return t11 + od * (1 - t11);
  }
  return 0.0;
}

/* One trajectory; returns EndSide (0 lost, 1 x-, 2 x+). */
__device__ int trace(const Geo64& g, const Task64& t, const Draw& rng, int64_t max_flights,
                     uint64_t* nflights, bool* capped, double* fpos) {
  const double X = g.box[0], Y = g.box[1], Z = g.box[2];
  double d0, d1, e0, e1;
  rng.block(0, 0, &d0, &d1);
  double pos[3] = {0.0, d0 * Y * g.scope[0], d1 * Z * g.scope[1]};
  rng.block(0, 1, &e0, &e1);
  double sphi, cphi;
  dsincos_2pi(e0, &sphi, &cphi);
  double dir[3] = {t.cth, t.sth * cphi, t.sth * sphi};
  int EndSide = (dir[0] <= 0.0) ? 1 : 0;
  int igrain = 0, isurf = 0, whichV = 0;
  if (g.kind_grain == 1) {
    double dmin = 1.0e10;
    for (int ig = 1; ig <= g.ngrain; ++ig) {
      if (!g.grain_incident[ig]) continue;
      const double* G = g.grain_gen + 3 * ig;
      const double a = pos[0] - G[0], b = pos[1] - G[1], c = pos[2] - G[2];
      const double d2 = a * a + b * b + c * c;
      if (dmin > d2) { dmin = d2; whichV = ig; }
    }
  } else {
    bool found = false;
    for (int ig = 1; ig <= g.ngrain; ++ig) {
      if (!g.grain_incident[ig]) continue;
      for (int k = g.grain_begin[ig]; k < g.grain_begin[ig + 1]; ++k) {
        if (!g.incident[k]) continue;
        if (in_polygon(g.vertex + 3 * (size_t)g.vbegin[k], g.nvertex[k], pos)) {
          whichV = ig;
          found = true;
          break;
        }
      }
    }
    if (!found) whichV = g.igrain_fill;
  }
  const bool ballistic = (t.lambda == kBallistic);
  double FreePath = ballistic ? kBallistic : -t.lambda * dlog_pos(e1);
  uint64_t flight = 0;
  *capped = false;
  while (EndSide == 0) {
    if (!(pos[0] >= 0.0 - kSmall && pos[0] <= X + kSmall && pos[1] >= 0.0 - kSmall &&
          pos[1] <= Y + kSmall && pos[2] >= 0.0 - kSmall && pos[2] <= Z + kSmall))
      break;
    if ((int64_t)flight >= max_flights) { *capped = true; break; }
    ++flight;
    const uint32_t fl = (uint32_t)flight;
    double distance = 1.0e10;
    int ig_min = igrain, is_min = isurf;
    for (int pass = 0; pass < 2; ++pass) {
      const int ig = pass == 0 ? 0 : whichV;
      if (pass == 1 && whichV == 0) break;
      const int kb = g.grain_begin[ig], ke = g.grain_begin[ig + 1];
      for (int k = kb; k < ke; ++k) {
        if (!g.internal[k]) continue;
        double L;
        if (surface_distance(g, k, pos, dir, &L) && distance > L) {
          distance = L;
          ig_min = ig;
          is_min = k - kb;
        }
      }
    }
    igrain = ig_min;
    isurf = is_min;
    int Jreflect = 1;
    bool pp = false;
    if (FreePath < distance) {
      distance = FreePath;
      for (int d = 0; d < 3; ++d) pos[d] = pos[d] + distance * dir[d];
      rng.block(fl, 0, &d0, &d1);
      const double ct = d0 * 2.0 - 1.0;
      double sp, cp;
      dsincos_2pi(d1, &sp, &cp);
      const double st = sqrt(1.0 - ct * ct);
      dir[0] = ct; dir[1] = st * cp; dir[2] = st * sp;
      igrain = 0;
      isurf = -1;
      pp = true;
    } else {
      for (int d = 0; d < 3; ++d) pos[d] = pos[d] + distance * dir[d];
      if (isurf < 0) {
        break;
      } else if (igrain == 0 && isurf == 0) {
        EndSide = 1;
      } else if (igrain == 0 && isurf == 1) {
        EndSide = 2;
      } else if (igrain == 0 && g.face_kind[isurf] == 1) {
        const int ax = isurf >> 1;
        if ((isurf & 1) == 0) pos[ax] = pos[ax] + g.box[ax];
        else pos[ax] = pos[ax] - g.box[ax];
      } else {
        const int k = g.grain_begin[igrain] + isurf;
        rng.block(fl, 0, &d0, &d1);
        double od = 0.0;
        if (g.nmaterial != 1 && (g.kind_trans[k] == 2 || g.kind_trans[k] == 3)) {
          double x;
          rng.block(fl, 2, &od, &x);
        }
        if (d0 <= g.spec[k]) {
          const double thr = threshold(g, k, t.omega, od);
          if (d1 <= thr) {
            Jreflect = 0;
          } else {
            double N[3];
            surface_normal(g, k, pos, N);
            if (dot3(N, dir) < 0) for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
            const double dn = dot3(N, dir);
            for (int d = 0; d < 3; ++d) dir[d] = dir[d] - 2.0 * N[d] * dn;
            Jreflect = 1;
          }
        } else {
          double N[3], Rm[9];
          surface_normal(g, k, pos, N);
          if (dot3(N, dir) < 0.0) for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
          surface_rotation(g, k, pos, Rm);
          double f0, f1;
          rng.block(fl, 1, &f0, &f1);
          const double sint = sqrt(d1);
          const double cost = sqrt(1.0 - sint * sint);
          double sp, cp;
          dsincos_2pi(f0, &sp, &cp);
          const double td[3] = {sint * cp, sint * sp, cost};
          double v[3];
          for (int i = 0; i < 3; ++i) v[i] = Rm[i] * td[0] + Rm[3 + i] * td[1] + Rm[6 + i] * td[2];
          if (dot3(dir, N) > 0.0) {
            for (int i = 0; i < 3; ++i) dir[i] = -v[i];
          } else {
            for (int i = 0; i < 3; ++i) dir[i] = v[i];
          }
          if (dot3(dir, N) > 0.0) for (int i = 0; i < 3; ++i) dir[i] = -1.0 * dir[i];
          const double thr = threshold(g, k, t.omega, od);
          if (f1 <= thr) {
            for (int i = 0; i < 3; ++i) dir[i] = -dir[i];
            Jreflect = 0;
          } else {
            Jreflect = 1;
          }
        }
      }
    }
    for (int d = 0; d < 3; ++d) pos[d] = pos[d] + 1.0e-7 * dir[d];
    if (ballistic) {
      FreePath = kBallistic;
    } else {
      FreePath = FreePath - distance;
      if (FreePath < 1.0e-10) {
        double r0, r1;
        if (pp) { rng.block(fl, 1, &r0, &r1); FreePath = -t.lambda * dlog_pos(r0); }
        else { rng.block(fl, 2, &r0, &r1); FreePath = -t.lambda * dlog_pos(r1); }
      }
    }
    if (Jreflect == 0) whichV = g.gout[g.grain_begin[igrain] + isurf];
  }
  *nflights = flight;
  if (fpos) { fpos[0] = pos[0]; fpos[1] = pos[1]; fpos[2] = pos[2]; }
  return EndSide;
}

__device__ __forceinline__ void warp_add_by_task(bool pred, long long task,
                                                 unsigned long long* arr) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (pred) {
    const unsigned peers = __match_any_sync(m, (unsigned long long)task);
    const int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) atomicAdd(arr + task, (unsigned long long)__popc(peers));
  }
}

__global__ void __launch_bounds__(128) k_plain_fp64(Geo64 g, Run64 r) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t task, j;
  if (r.replay_task >= 0) {
    task = r.replay_task;
    j = gid;
  } else {
    task = gid / r.np_local;
    j = gid - task * r.np_local;
  }
  const bool active = (r.replay_task >= 0) ? (gid < r.np_local) : (task < r.ntask);
  int es = -1;
  uint64_t nf = 0;
  bool capped = false;
  bool run = false;
  if (active) {
    const Task64 t = r.task[task];
    if (t.lambda > 0.0) {
      run = true;
      const int64_t p = r.rank + j * (int64_t)r.nranks;
      const uint64_t sample = (uint64_t)task * (uint64_t)r.np + (uint64_t)p;
      Draw rng;
      rng.key.k0 = r.k0;
      rng.key.k1 = r.k1;
      rng.c1 = r.c1;
      rng.slo = (uint32_t)sample;
      rng.shi = (uint32_t)(sample >> 32);
      double fp[3];
      es = trace(g, t, rng, r.max_flights, &nf, &capped, fp);
      if (r.replay_task >= 0) {
        r.end_side[j] = es;
        r.flights[j] = (unsigned)nf;
        r.final_pos[3 * j] = fp[0];
        r.final_pos[3 * j + 1] = fp[1];
        r.final_pos[3 * j + 2] = fp[2];
      }
    } else if (r.replay_task >= 0) {
      r.end_side[j] = 0;
      r.flights[j] = 0;
      r.final_pos[3 * j] = r.final_pos[3 * j + 1] = r.final_pos[3 * j + 2] = 0.0;
    }
  }
  const bool trans = run && (es == 2 || (es == 0 && r.ref_quirks));
  const bool lostp = run && es == 0;
  warp_add_by_task(trans, task, r.counts);
  warp_add_by_task(lostp, task, r.lost);
  /* warp totals of flights / lost / capped / samples */
  unsigned long long v0 = nf, v1 = lostp, v2 = capped, v3 = run;
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
    v3 += __shfl_xor_sync(0xffffffffu, v3, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (v0) atomicAdd(r.stats + 0, v0);
    if (v1) atomicAdd(r.stats + 1, v1);
    if (v2) atomicAdd(r.stats + 2, v2);
    if (v3) atomicAdd(r.stats + 3, v3);
  }
}

}  // namespace

cudaError_t launch_plain_fp64(const Geo64& g, const Run64& r, cudaStream_t st, int* grid_out,
                              int* block_out) {
  const int block = 128;
  const int64_t nthreads = (r.replay_task >= 0) ? r.np_local : r.ntask * r.np_local;
  if (nthreads <= 0) return cudaSuccess;
  const int64_t grid = (nthreads + block - 1) / block;
  if (grid > 2147483647LL) return cudaErrorInvalidConfiguration;
  k_plain_fp64<<<(unsigned)grid, block, 0, st>>>(g, r);
  if (grid_out) *grid_out = (int)grid;
  if (block_out) *block_out = block;
  return cudaGetLastError();
}

}  // namespace ptg
