/*
 * gamma.cpp - ptg_gamma_from_tbc: the interface parameter gamma of a TBC
 * transmission entry.
 *
 * A "TBC" entry of the .mcp transmission table gives a thermal boundary
 * conductance G; the reference turns it into the gamma of the per-mode
 * transmissivity T(omega) = 1 / (gamma * omega / omega_max + 1)
 * (setupSurfaceTransmissivity, src/RTMCphon.f90:1402-1429) by Newton's
 * method on F(gamma) = G_T / (1 - G_T / G_1) - G, where
 * G_T = sum_modes w C v T / (2 vol nqfbz) and G_1 the same sum with T = 1
 * (GammaDeterm, :2499-2599): start at gamma = 1e-2, at most 10000 steps,
 * stop when |F / F'| <= 1e-6.  The sums run over the material's modes in
 * the reference's order (k-point outer, branch inner) with its constants.
 */
#include <cmath>
#include <string>

#include "ptg_internal.h"

extern "C" int ptg_gamma_from_tbc(const ptg_spectrum* material, double temperature, double tbc,
                                  double* gamma) {
  if (!material || !gamma || !(temperature > 0.0)) return PTG_ERR_INVALID;
  std::string why;
  ptg::SpecSoA S;
  if (ptg::copy_spectrum(material, &S, &why) != PTG_OK) return PTG_ERR_INVALID;
  const double hbar = 1.054571e-34, kB = 1.3806503e-23;  /* src/RTMCphon.f90:66-67 */
  const int nb = S.nb, nk = S.nk;
  auto M = [&](int kk, int jj) { return (size_t)kk + (size_t)nb * jj; };
  double wsum = 0.0;
  for (int jj = 0; jj < nk; ++jj)
    for (int kk = 0; kk < nb; ++kk) wsum += S.weight[M(kk, jj)];
  const int nqfbz = (int)(wsum / nb);
  std::vector<double> cap((size_t)nb * nk);
  for (int ii = 0; ii < nk; ++ii)
    for (int jj = 0; jj < nb; ++jj) {
      const double x = hbar * S.omega[M(jj, ii)] / (kB * temperature);
      if (x <= 1.0e-10) cap[M(jj, ii)] = kB;
      else {
        const double q = (x / 2) / sinh(x / 2);
        cap[M(jj, ii)] = kB * (q * q);
      }
    }
  const double wmax = S.max_omega;
  double g = 1.0e-2;
  for (int it = 0; it < 10000; ++it) {
    double t = 0.0, ta = 0.0, dt = 0.0;
    for (int jj = 0; jj < nk; ++jj)
      for (int kk = 0; kk < nb; ++kk) {
        const size_t m = M(kk, jj);
        const double h = 1 / (g * (S.omega[m] / wmax) + 1);
        t = t + S.weight[m] * cap[m] * S.vel[m] * h / 2 / S.vol / nqfbz;
      }
    for (int jj = 0; jj < nk; ++jj)
      for (int kk = 0; kk < nb; ++kk) {
        const size_t m = M(kk, jj);
        const double h = 1;
        ta = ta + S.weight[m] * cap[m] * S.vel[m] * h / 2 / S.vol / nqfbz;
      }
    for (int jj = 0; jj < nk; ++jj)
      for (int kk = 0; kk < nb; ++kk) {
        const size_t m = M(kk, jj);
        const double r = g * (S.omega[m] / wmax) + 1;
        const double h = -(S.omega[m] / wmax) / (r * r);
        dt = dt + S.weight[m] * cap[m] * S.vel[m] * h / 2 / S.vol / nqfbz;
      }
    const double F = t / (1 - t / ta) - tbc;
    const double q = 1 - t / ta;
    const double dF = dt / (q * q);
    const double step = F / dF;
    if (std::fabs(step) <= 1.0e-6) break;
    g = g - step;
  }
  *gamma = g;
  return g < 0.0 ? PTG_ERR_INVALID : PTG_OK;
}
