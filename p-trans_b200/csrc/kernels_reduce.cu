/*
 * kernels_reduce.cu - FP64 reduction from transmitted counts to effective
 * MFPs, kappa and the per-frequency-bin transmission.
 *
 * Per mode (one thread): Simpson's rule over the incident angle
 * (effectiveMFP, src/RTMCphon.f90:2418-2451), the effective MFP rule of
 * fileoutput (Matthiessen :2715-2719, grid interpolation :2722-2744, or the
 * mode's own MFP), kappa_mode = K_m * EMFP (:2747-2749) and the binomial
 * variance of every term.  Then one block sums kappa in a fixed tree order and
 * one block per frequency bin sums its flux-weighted transmission, so the
 * result does not depend on scheduling.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace ptg {

namespace {

/* Per-mode terms of one geometry; the batched kernel calls it with the
   geometry's counts, np, Simpson step and output rows. */
__device__ void mode_terms(const ReduceIn& in, int64_t m) {
  const int na = in.nangle, ns = in.ns;
  double S[64], V[64], dE[64];
  /* ns <= 64 is checked on the host */
  for (int s = 0; s < ns; ++s) {
    double acc = 0.0, var = 0.0;
    for (int ia = 0; ia < na - 1; ++ia) {
      const int64_t task = m + in.nmode * (s + (int64_t)ns * ia);
      const double tr = (double)in.counts[task] / in.np;
      const double c = in.coef[ia];
      acc += c * tr;
      var += c * c * (tr * (1.0 - tr) / in.np);
      if (in.transmit) in.transmit[task] = tr;
    }
    if (in.transmit) in.transmit[m + in.nmode * (s + (int64_t)ns * (na - 1))] = 0.0;
    S[s] = acc * in.dS;
    V[s] = var * in.dS * in.dS;
    dE[s] = 0.0;
  }
  const double mf = in.mfp_m[m];
  double E;
  if (in.kind_mfp == 1) {
    if (mf == 0.0) {
      E = S[0] * 1.0e-9;
      dE[0] = 1.0e-9;
    } else {
      const double sm = S[0] * 1.0e-9;
      E = 1.0 / (1.0 / mf + 1.0 / sm);
      dE[0] = (sm > 0.0) ? 1.0e-9 * (E * E) / (sm * sm) : 1.0e-9;
    }
  } else if (in.kind_mfp == 3) {
    E = S[0] * 1.0e-9;
    dE[0] = 1.0e-9;
  } else {
    const double* g = in.grid;
    if (mf < g[0] * 1.0e-9) {
      E = S[0] * 1.0e-9 * mf / (g[0] * 1.0e-9);
      dE[0] = 1.0e-9 * mf / (g[0] * 1.0e-9);
    } else if (mf > g[ns - 1] * 1.0e-9) {
      E = S[ns - 1] * 1.0e-9;
      dE[ns - 1] = 1.0e-9;
    } else {
      E = S[ns - 1] * 1.0e-9;
      dE[ns - 1] = 1.0e-9;
      for (int s = 0; s < ns - 1; ++s) {
        if (g[s] * 1.0e-9 <= mf && mf < g[s + 1] * 1.0e-9) {
          const double ip = (mf - g[s] * 1.0e-9) / ((g[s + 1] - g[s]) * 1.0e-9);
          E = S[s] * 1.0e-9 * (1.0 - ip) + S[s + 1] * 1.0e-9 * ip;
          dE[ns - 1] = 0.0;
          dE[s] = 1.0e-9 * (1.0 - ip);
          dE[s + 1] = 1.0e-9 * ip;
          break;
        }
      }
    }
  }
  const double K = in.K[m];
  double kv = 0.0;
  for (int s = 0; s < ns; ++s) {
    const double gk = K * dE[s];
    kv += gk * gk * V[s];
  }
  in.tc[m] = K * E;
  in.kv[m] = kv;
  in.emfp_nm[m] = E * 1.0e9;
  /* per-bin transmission <T> = EMFP / (0.75 Lx) (ballistic <T> for Matthiessen) */
  double tm, vm = 0.0;
  if (in.kind_mfp == 1) {
    tm = S[0] / in.tnorm;
    vm = V[0] / (in.tnorm * in.tnorm);
  } else {
    tm = E * 1.0e9 / in.tnorm;
    for (int s = 0; s < ns; ++s) {
      const double gk = dE[s] * 1.0e9 / in.tnorm;
      vm += gk * gk * V[s];
    }
  }
  const double W = in.W[m];
  in.bw[m] = W * tm;
  in.bv[m] = W * W * vm;
}

__global__ void k_mode_terms(ReduceIn in) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= in.nmode) return;
  mode_terms(in, m);
}

__global__ void k_mode_terms_batch(ReduceBatchIn b) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (m >= b.base.nmode) return;
  ReduceIn in = b.base;
  const int64_t nm = in.nmode;
  in.counts = b.base.counts + (int64_t)g * b.ntask_per_geo;
  in.np = b.np_geo[g];
  in.dS = b.dS_geo[g];
  in.tnorm = b.tnorm_geo[g];
  in.tc = b.base.tc + g * nm;
  in.kv = b.base.kv + g * nm;
  in.bw = b.base.bw + g * nm;
  in.bv = b.base.bv + g * nm;
  in.emfp_nm = b.base.emfp_nm + g * nm;
  in.transmit = nullptr;
  mode_terms(in, m);
}

/* block 0: kappa and its variance; block 1+b: bin b. Fixed-order sums. */
__device__ void sums(const ReduceIn& in, int b) {
  __shared__ double sh[3][1024];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t m = threadIdx.x; m < in.nmode; m += blockDim.x) {
    if (b < 0) {
      a0 += in.tc[m];
      a1 += in.kv[m];
    } else if (in.bin[m] == b) {
      a0 += in.W[m];
      a1 += in.bw[m];
      a2 += in.bv[m];
    }
  }
  sh[0][threadIdx.x] = a0;
  sh[1][threadIdx.x] = a1;
  sh[2][threadIdx.x] = a2;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (b < 0) {
      in.result[0] = sh[0][0];
      in.result[1] = sh[1][0];
    } else {
      in.result[2 + 3 * b] = sh[0][0];
      in.result[3 + 3 * b] = sh[1][0];
      in.result[4 + 3 * b] = sh[2][0];
    }
  }
}

__global__ void __launch_bounds__(1024) k_sums(ReduceIn in) { sums(in, (int)blockIdx.x - 1); }

__global__ void __launch_bounds__(1024) k_sums_batch(ReduceBatchIn bi) {
  ReduceIn in = bi.base;
  const int g = blockIdx.y;
  const int64_t nm = in.nmode;
  in.tc = bi.base.tc + g * nm;
  in.kv = bi.base.kv + g * nm;
  in.bw = bi.base.bw + g * nm;
  in.bv = bi.base.bv + g * nm;
  in.result = bi.base.result + (int64_t)g * (2 + 3 * in.nbins);
  sums(in, (int)blockIdx.x - 1);
}

}  // namespace

cudaError_t launch_kappa_reduce(const ReduceIn& in, cudaStream_t st) {
  if (in.nmode <= 0) return cudaSuccess;
  if (in.ns > 64) return cudaErrorInvalidValue;
  const int block = 128;
  const int64_t grid = (in.nmode + block - 1) / block;
  k_mode_terms<<<(unsigned)grid, block, 0, st>>>(in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sums<<<1 + in.nbins, 1024, 0, st>>>(in);
  return cudaGetLastError();
}

cudaError_t launch_kappa_reduce_batch(const ReduceBatchIn& b, cudaStream_t st) {
  if (b.base.nmode <= 0 || b.ngeo <= 0) return cudaSuccess;
  if (b.base.ns > 64 || b.ngeo > 65535) return cudaErrorInvalidValue;
  const int block = 128;
  dim3 g1((unsigned)((b.base.nmode + block - 1) / block), (unsigned)b.ngeo);
  k_mode_terms_batch<<<g1, block, 0, st>>>(b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 g2((unsigned)(1 + b.base.nbins), (unsigned)b.ngeo);
  k_sums_batch<<<g2, 1024, 0, st>>>(b);
  return cudaGetLastError();
}

}  // namespace ptg
