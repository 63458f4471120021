/*
 * writers.cpp - ptg_write_outputs: the reference's result files from the
 * transmitted counts of a run.
 *
 * fileoutput (src/RTMCphon.f90:2601-2881) writes, next to the .mcp file,
 *   thermalproperty.out      incident phonons, averaged effective MFP, kappa
 *   effectiveMFP.out         per mode: branch, k-point, bulk and effective MFP,
 *                            kappa and its running sum, by effective MFP
 *   phononconductivity.out   kappa per distinct frequency and branch
 * from SEMFP (effectiveMFP, :2418-2451).  The numbers are formed in the
 * reference's order (Simpson sum, per-branch exchange sort by omega, column
 * major sums) and printed with its edit descriptors (i, f, e as gfortran
 * writes them: 0.ddddE+xx mantissas, asterisks on overflow), so the files
 * read the same as the reference's for the same SEMFP.  The orderings use
 * O(n log n) sorts when the keys are distinct; with ties they fall back to
 * the reference's exchange sorts, whose placement of equal keys is part of
 * the output.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ptg_internal.h"

namespace {

/* the reference's constants, src/RTMCphon.f90:61-67 */
constexpr double kHbar = 1.054571e-34;
constexpr double kKB = 1.3806503e-23;
constexpr double kPi = 3.14159265358979323846;

std::string pad_left(const std::string& s, int w) {
  if (w <= 0 || (int)s.size() >= w) return s;
  return std::string(w - s.size(), ' ') + s;
}

/* Iw */
std::string fort_i(long long v, int w) {
  std::string s = std::to_string(v);
  if ((int)s.size() > w) return std::string(w, '*');
  return pad_left(s, w);
}

/* Fw.d (w = 0: minimal width) */
std::string fort_f(double v, int w, int d) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%.*f", d, v);
  std::string s = buf;
  if (w == 0) return s;
  if ((int)s.size() > w) {
    /* the optional leading zero goes first */
    if (s.rfind("0.", 0) == 0) s = s.substr(1);
    else if (s.rfind("-0.", 0) == 0) s = "-" + s.substr(2);
    if ((int)s.size() > w) return std::string(w, '*');
  }
  return pad_left(s, w);
}

/* Ew.d: [-]0.d1..dd E+xx (|exp| <= 99) or [-]0.d1..dd+xxx */
std::string fort_e(double v, int w, int d) {
  std::string mant, ex;
  const bool neg = std::signbit(v) && v != 0.0;
  int e10 = 0;
  if (v == 0.0) {
    mant = std::string(d, '0');
  } else {
    char buf[128];
    snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));
    const char* p = buf;
    mant.push_back(p[0]);
    const char* q = strchr(p, '.');
    const char* e = strchr(p, 'e');
    if (q) mant.append(q + 1, e - q - 1);
    e10 = atoi(e + 1) + 1;
  }
  char eb[16];
  if (std::abs(e10) <= 99) snprintf(eb, sizeof(eb), "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
  else snprintf(eb, sizeof(eb), "%c%03d", e10 < 0 ? '-' : '+', std::abs(e10));
  std::string s = std::string(neg ? "-" : "") + "0." + mant + eb;
  if ((int)s.size() > w) {
    s = std::string(neg ? "-" : "") + "." + mant + eb;
    if ((int)s.size() > w) return std::string(w, '*');
  }
  return pad_left(s, w);
}

/* The reference's exchange sort: for each position the first minimum of the
   rest arrives there by swaps.  key(i) < key(j) decides; swap(i, j) moves
   whole records. */
template <class Key, class Swap>
void exchange_sort(int n, Key key, Swap swp) {
  for (int i = 0; i < n - 1; ++i)
    for (int j = i + 1; j < n; ++j)
      if (key(i) > key(j)) swp(i, j);
}

/* Ascending order of keys; an exchange sort when two keys are equal (the
   reference's tie placement), else a permutation sort. Returns the order. */
std::vector<int> reference_order(const std::vector<double>& keys) {
  const int n = (int)keys.size();
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::vector<double> sorted = keys;
  std::sort(sorted.begin(), sorted.end());
  bool ties = false;
  for (int i = 1; i < n; ++i)
    if (sorted[i] == sorted[i - 1]) { ties = true; break; }
  if (!ties) {
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    return idx;
  }
  std::vector<double> k = keys;
  exchange_sort(
      n, [&](int i) { return k[i]; },
      [&](int i, int j) {
        std::swap(k[i], k[j]);
        std::swap(idx[i], idx[j]);
      });
  return idx;
}

bool write_text(const std::string& path, const std::string& text) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  const bool ok = fwrite(text.data(), 1, text.size(), f) == text.size();
  return fclose(f) == 0 && ok;
}

}  // namespace

extern "C" int ptg_write_outputs(const char* geofile, const ptg_geometry* geom,
                                 const ptg_spectrum* spec, const ptg_run* run,
                                 const uint64_t* counts) {
  try {
    if (!geofile || !geom || !spec || !run || !counts) return PTG_ERR_INVALID;
    std::string why;
    ptg::SpecSoA S;
    if (ptg::copy_spectrum(spec, &S, &why) != PTG_OK) return PTG_ERR_INVALID;
    if (!ptg::run_valid(S, run, &why)) return PTG_ERR_INVALID;
    const int nb = S.nb, nk = S.nk, na = run->nangle;
    const int ns = run->kind_mfp == PTG_MFP_GRID ? run->nmfp : 1;
    const int64_t nm = (int64_t)nb * nk;
    const double T = run->temperature;
    const double boxx = geom->box[0];
    /* SEMFP(ik, ib, s): effectiveMFP, :2418-2446 */
    std::vector<double> vangle(na);
    for (int ia = 0; ia < na; ++ia)
      vangle[ia] = 0.0 + (double)ia / (double)(na - 1) * (kPi * 0.5);
    const double dS = (vangle[1] - vangle[0]) / 3.0 * 3.0 * 0.5 * boxx;
    auto SE = [&](int ik, int ib, int s) -> size_t { return (size_t)ik + (size_t)nk * (ib + (size_t)nb * s); };
    std::vector<double> semfp((size_t)nm * ns), WT(na);
    for (int s = 0; s < ns; ++s)
      for (int ik = 0; ik < nk; ++ik)
        for (int ib = 0; ib < nb; ++ib) {
          const int64_t m = ib + (int64_t)nb * ik;
          for (int ia = 0; ia < na; ++ia) {
            double tr = 0.0;
            if (ia < na - 1) tr = (double)counts[m + nm * (s + (int64_t)ns * ia)] / (double)run->np;
            WT[ia] = sin(vangle[ia]) * cos(vangle[ia]) * tr;
          }
          double I = 0.0;
          for (int ia = 1; ia < na - 1; ia += 2) I = I + (WT[ia - 1] + 4.0 * WT[ia] + WT[ia + 1]);
          semfp[SE(ik, ib, s)] = I * dS;
        }
    /* output directory: GeoFile up to its last separator, :2629-2632 */
    std::string gf = geofile;
    size_t cut = gf.find_last_of('/');
    if (cut == std::string::npos) cut = gf.find_last_of('\\');
    const std::string dir = (cut == std::string::npos) ? std::string() : gf.substr(0, cut + 1);
  
    std::string tp;
    tp += "# Datatype = thermalproperty\n";
    tp += "# Incident_Phonon                               =   " + fort_i(run->np, 6) + "\n";
    if (geom->nmaterial > 1) {
      tp += "# Effective_MeanFreePath [nm]       = " + fort_e(semfp[SE(0, 0, 0)], 20, 10) + "\n";
      return write_text(dir + "thermalproperty.out", tp) ? PTG_OK : PTG_ERR_IO;
    }
    double sum = 0.0;
    for (size_t i = 0; i < semfp.size(); ++i) sum += semfp[i];
    const double ave = sum / (double)(nb * nk * ns);
    tp += "# Averaged Effective_MeanFreePath [nm]          = " + fort_f(ave, 20, 10) + "\n";
  
    /* mode arrays (branch, k-point), rescaled tau and bulk MFP, :2642-2647 */
    const double scale = run->scatter_scale > 0.0 ? run->scatter_scale : 1.0;
    auto M = [&](int ib, int ik) -> size_t { return (size_t)ib + (size_t)nb * ik; };
    std::vector<double> om(S.omega), wt(S.weight), ta(S.tau), ve(S.vel), mf(nm);
    for (int64_t m = 0; m < nm; ++m) {
      ta[m] = ta[m] * 1.0e-12 * (S.rtemp / T);
      mf[m] = ta[m] * ve[m] / scale;
    }
    double wsum = 0.0;
    for (int64_t m = 0; m < nm; ++m) wsum += wt[m];
    const int nqfbz = (int)(wsum / nb);
    /* per-branch order by omega, :2658-2691 (SEMFP travels along) */
    for (int ib = 0; ib < nb; ++ib) {
      std::vector<double> key(nk);
      for (int ik = 0; ik < nk; ++ik) key[ik] = om[M(ib, ik)];
      const std::vector<int> ord = reference_order(key);
      std::vector<double> o2(nk), w2(nk), t2(nk), v2(nk), m2(nk), s2((size_t)nk * ns);
      for (int i = 0; i < nk; ++i) {
        const int src = ord[i];
        o2[i] = om[M(ib, src)]; w2[i] = wt[M(ib, src)]; t2[i] = ta[M(ib, src)];
        v2[i] = ve[M(ib, src)]; m2[i] = mf[M(ib, src)];
        for (int s = 0; s < ns; ++s) s2[(size_t)i * ns + s] = semfp[SE(src, ib, s)];
      }
      for (int i = 0; i < nk; ++i) {
        om[M(ib, i)] = o2[i]; wt[M(ib, i)] = w2[i]; ta[M(ib, i)] = t2[i];
        ve[M(ib, i)] = v2[i]; mf[M(ib, i)] = m2[i];
        for (int s = 0; s < ns; ++s) semfp[SE(i, ib, s)] = s2[(size_t)i * ns + s];
      }
    }
    /* heat capacity, effective MFP rule and kappa per mode, :2693-2751 */
    std::vector<double> cap(nm), emfp(nm), tc(nm);
    for (int ib = 0; ib < nb; ++ib)
      for (int ik = 0; ik < nk; ++ik) {
        const size_t m = M(ib, ik);
        const double x = kHbar * om[m] / (kKB * T);
        if (x <= 1.0e-10) cap[m] = kKB;
        else {
          const double q = (x / 2) / sinh(x / 2);
          cap[m] = kKB * (q * q);
        }
        double E;
        const double s0 = semfp[SE(ik, ib, 0)];
        if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
          if (mf[m] == 0.0) E = s0 * 1.0e-9;
          else E = 1.0 / (1.0 / mf[m] + 1.0 / (s0 * 1.0e-9));
        } else if (run->kind_mfp == PTG_MFP_PER_MODE) {
          E = s0 * 1.0e-9;
        } else {
          const double* g = run->mfp_grid_nm;
          if (mf[m] < g[0] * 1.0e-9) {
            E = s0 * 1.0e-9 * mf[m] / (g[0] * 1.0e-9);
          } else if (mf[m] > g[ns - 1] * 1.0e-9) {
            E = semfp[SE(ik, ib, ns - 1)] * 1.0e-9;
          } else {
            /* mf equal to the last grid point matches no interval (the
               reference leaves EMFP unset there): the last SEMFP */
            E = semfp[SE(ik, ib, ns - 1)] * 1.0e-9;
            for (int s = 0; s < ns - 1; ++s) {
              if (g[s] * 1.0e-9 <= mf[m] && mf[m] < g[s + 1] * 1.0e-9) {
                const double ip = (mf[m] - g[s] * 1.0e-9) / ((g[s + 1] - g[s]) * 1.0e-9);
                E = semfp[SE(ik, ib, s)] * 1.0e-9 * (1.0 - ip) + semfp[SE(ik, ib, s + 1)] * 1.0e-9 * ip;
                break;
              }
            }
          }
        }
        emfp[m] = E;
        tc[m] = cap[m] * wt[m] * E * ve[m] / 3 / S.vol / nqfbz;
      }
    double kappa = 0.0;
    for (int ik = 0; ik < nk; ++ik)
      for (int ib = 0; ib < nb; ++ib) kappa += tc[M(ib, ik)];
    tp += "# Thermal_conductivity@" + fort_f(T, 0, 6) + "K [W m-1 K-1]  = " + fort_f(kappa, 20, 10) + "\n";
    if (!write_text(dir + "thermalproperty.out", tp)) return PTG_ERR_IO;
  
    /* effectiveMFP.out, :2756-2809: records (branch-major) by effective MFP */
    const int cfreq = (int)nm;
    std::vector<int> rb(cfreq), rk(cfreq);
    std::vector<double> key(cfreq);
    {
      int kk = 0;
      for (int ib = 0; ib < nb; ++ib)
        for (int ik = 0; ik < nk; ++ik, ++kk) {
          rb[kk] = ib;
          rk[kk] = ik;
          key[kk] = emfp[M(ib, ik)];
        }
    }
    const std::vector<int> ord = reference_order(key);
    std::string em;
    em += "# Datatype = Effective Mean Free Path of phonon.\n";
    em += "# data are sorted by effective MFP in ascending order.\n";
    em += "#   total branches: " + fort_i(nb, 3) + "\n";
    em += "#   total Kpoints:  " + fort_i(nk, 3) + "\n";
    em += "#\n";
    em += "# branch, kpoint, bulk MFP[nm], effective MFP[nm], ThermalConductivity, and its "
          "accumulated[W m-1 K-1].\n";
    double accum = 0.0;
    for (int i = 0; i < cfreq; ++i) {
      const int r = ord[i];
      const size_t m = M(rb[r], rk[r]);
      accum = (i == 0) ? tc[m] : tc[m] + accum;
      em += fort_i(rb[r] + 1, 5) + fort_i(rk[r] + 1, 5) + fort_e(mf[m] * 1.0e9, 15, 6) +
            fort_e(emfp[m] * 1.0e9, 15, 6) + fort_e(tc[m], 15, 6) + fort_e(accum, 15, 6) + "\n";
    }
    if (!write_text(dir + "effectiveMFP.out", em)) return PTG_ERR_IO;
  
    /* phononconductivity.out, :2811-2865: distinct frequencies, ascending;
       the largest is left out (the loop runs to cfreq-1) */
    std::vector<double> freq;
    for (int ib = 0; ib < nb; ++ib)
      for (int ik = 0; ik < nk; ++ik) {
        const double w = om[M(ib, ik)];
        if (std::find(freq.begin(), freq.end(), w) == freq.end()) freq.push_back(w);
      }
    std::sort(freq.begin(), freq.end());
    const int nf = (int)freq.size();
    std::string pc;
    pc += "# Datatype = phononconductivity\n";
    pc += "# Nb = " + fort_i(nf - 1, 6) + "\n";
    pc += "# Nbranch = " + fort_i(nb, 4) + "\n";
    pc += "# omega, fluxphononout(1:Nbranch)\n";
    for (int i = 0; i < nf - 1; ++i) {
      pc += fort_e(freq[i], 20, 10);
      for (int ib = 0; ib < nb; ++ib) {
        double k = 0.0;
        for (int ik = 0; ik < nk; ++ik)
          if (om[M(ib, ik)] == freq[i]) k = k + tc[M(ib, ik)];
        pc += fort_e(k, 20, 10);
      }
      pc += "\n";
    }
    if (!write_text(dir + "phononconductivity.out", pc)) return PTG_ERR_IO;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    return PTG_ERR_NOMEM;
  } catch (...) {
    return PTG_ERR_INVALID;
  }
}

/* Fortran edit-descriptor formatting, exported for the tests of the writer
   (kind 0: Iw, 1: Fw.d, 2: Ew.d).  Writes at most cap bytes with a NUL. */
extern "C" int ptg_fortran_format(int32_t kind, double v, int32_t w, int32_t d, char* out,
                                  int32_t cap) {
  if (!out || cap < 1) return PTG_ERR_INVALID;
  std::string s;
  if (kind == 0) s = fort_i((long long)v, w);
  else if (kind == 1) s = fort_f(v, w, d);
  else if (kind == 2) s = fort_e(v, w, d);
  else return PTG_ERR_INVALID;
  if ((int)s.size() + 1 > cap) return PTG_ERR_INVALID;
  memcpy(out, s.c_str(), s.size() + 1);
  return PTG_OK;
}
