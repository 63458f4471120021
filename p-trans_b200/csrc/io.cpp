/*
 * io.cpp - readers for the reference's input files.
 *
 *   .mcp     loadMCP and its loaders, src/RTMCphon.f90:252-1251: every scalar
 *            parameter is found by scanning for a line whose first token is
 *            the key (findKey, :212-231) and reading the next line; the
 *            material, transmission-table and grain sections are then read
 *            line by line in the reference's order.
 *   .anphon  loadAnphon, src/RTMCphon.f90:661-733 (omega converted from
 *            cm^-1 with 0.03 THz per cm^-1 and 2*pi*1e12), and a writer of
 *            the same layout for synthetic spectra.
 *
 * Tokens are separated by blanks or commas, like Fortran list-directed input;
 * a numeric read takes the leading tokens and ignores the rest of the line.
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "ptg_internal.h"

namespace {

std::vector<std::string> tokens(const std::string& line) {
  std::vector<std::string> out;
  std::string cur;
  for (char ch : line) {
    if (isspace((unsigned char)ch) || ch == ',') {
      if (!cur.empty()) { out.push_back(cur); cur.clear(); }
    } else {
      cur.push_back(ch);
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

bool to_double(const std::string& s, double* v) {
  std::string t = s;
  for (char& c : t) if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  *v = strtod(t.c_str(), &end);
  return end && *end == '\0' && !t.empty();
}

bool to_int(const std::string& s, long long* v) {
  char* end = nullptr;
  *v = strtoll(s.c_str(), &end, 10);
  return end && *end == '\0' && !s.empty();
}

struct Lines {
  std::vector<std::string> l;
  size_t pos = 0;
  /* findKey: first line (from the top) whose first token equals key; the
     cursor is left on the following line */
  bool find(const std::string& key) {
    for (size_t i = 0; i < l.size(); ++i) {
      std::vector<std::string> t = tokens(l[i]);
      if (t.empty()) continue;
      if (t[0] == key) { pos = i + 1; return true; }
    }
    return false;
  }
  bool next(std::string* s) {
    if (pos >= l.size()) return false;
    *s = l[pos++];
    return true;
  }
};

bool read_doubles(const std::string& line, int n, double* v) {
  std::vector<std::string> t = tokens(line);
  if ((int)t.size() < n) return false;
  for (int i = 0; i < n; ++i)
    if (!to_double(t[i], &v[i])) return false;
  return true;
}

bool read_int(const std::string& line, long long* v) {
  std::vector<std::string> t = tokens(line);
  return !t.empty() && to_int(t[0], v);
}

}  // namespace

struct ptg_mcpbuf {
  ptg_model m;
  std::vector<int32_t> tt_kind, grain_shape, grain_material, grain_nfacet, facet_nvertex,
      surf_material_to, surf_grain_to;
  std::vector<double> tt_trans, tt_spec, grain_generatrix, grain_diameter, facet_vertex;
  std::vector<std::string> materials;
  std::vector<double> mfp_grid;
  int64_t np = 0;
  int32_t nangle = 91, kind_mfp = PTG_MFP_MATTHIESSEN, particle_trace = 1000;
};

namespace {

int parse_mcp(Lines& L, ptg_mcpbuf* b) {
  ptg_model& m = b->m;
  memset(&m, 0, sizeof(m));
  std::string line;
  long long iv;
  double dv;
  /* loadParameterBox, src/RTMCphon.f90:279-420 */
  long long N[3];
  const char* nk[3] = {"NXcell", "NYcell", "NZcell"};
  const char* lk[3] = {"LXcell", "LYcell", "LZcell"};
  for (int d = 0; d < 3; ++d) {
    if (!L.find(nk[d]) || !L.next(&line) || !read_int(line, &N[d])) return PTG_ERR_IO;
  }
  for (int d = 0; d < 3; ++d) {
    if (!L.find(lk[d]) || !L.next(&line) || !read_doubles(line, 1, &dv)) return PTG_ERR_IO;
    m.box[d] = dv * (double)N[d];
  }
  if (!L.find("CellSpecularity")) {
    for (int f = 0; f < 6; ++f) m.cellspec[f] = 1.0;
  } else {
    if (!L.next(&line)) return PTG_ERR_IO;
    if (!read_doubles(line, 6, m.cellspec)) {
      if (!read_doubles(line, 1, &dv)) return PTG_ERR_IO;
      for (int f = 0; f < 6; ++f) m.cellspec[f] = dv;
    }
  }
  m.specfluc = 0.0;
  if (L.find("FluctuationSpecularity")) {
    if (!L.next(&line) || !read_doubles(line, 1, &m.specfluc)) return PTG_ERR_IO;
  }
  /* loadParameterPhonon, :424-589 */
  if (!L.find("temp") || !L.next(&line) || !read_doubles(line, 1, &m.temperature)) return PTG_ERR_IO;
  if (!L.find("Np") || !L.next(&line) || !read_int(line, &iv)) return PTG_ERR_IO;
  b->np = iv;
  b->nangle = 91;
  if (L.find("Nangle")) {
    if (!L.next(&line) || !read_int(line, &iv)) return PTG_ERR_IO;
    b->nangle = (int32_t)iv;
  }
  m.scope[0] = m.scope[1] = 1.0;
  if (L.find("ScopeY") && (!L.next(&line) || !read_doubles(line, 1, &m.scope[0]))) return PTG_ERR_IO;
  if (L.find("ScopeZ") && (!L.next(&line) || !read_doubles(line, 1, &m.scope[1]))) return PTG_ERR_IO;
  if (!L.find("MeanFreePath")) {
    b->kind_mfp = PTG_MFP_MATTHIESSEN;
    b->mfp_grid.assign(1, 1.0e10);
  } else {
    b->kind_mfp = PTG_MFP_GRID;
    if (!L.next(&line)) return PTG_ERR_IO;
    std::vector<std::string> t = tokens(line);
    double lo, hi;
    long long n;
    if (t.size() >= 4 && to_double(t[0], &lo) && to_double(t[1], &hi) && to_int(t[2], &n)) {
      if (lo < 0.0 || lo > hi || n <= 0) return PTG_ERR_IO;
      b->mfp_grid.resize(n);
      if (t[3] == "linear") {
        for (long long s = 0; s < n; ++s)
          b->mfp_grid[s] = n > 1 ? lo + (hi - lo) / (double)(n - 1) * (double)s : lo;
      } else if (t[3] == "log") {
        for (long long s = 0; s < n; ++s)
          b->mfp_grid[s] = n > 1 ? exp(log(lo) + (log(hi) - log(lo)) / (double)(n - 1) * (double)s) : lo;
      } else {
        return PTG_ERR_IO;
      }
    } else {
      if (!read_doubles(line, 1, &lo) || lo < 0.0) return PTG_ERR_IO;
      b->mfp_grid.assign(1, lo);
    }
  }
  b->particle_trace = 1000;
  if (L.find("Trace")) {
    if (!L.next(&line) || !read_int(line, &iv)) return PTG_ERR_IO;
    b->particle_trace = (int32_t)iv;
  }
  /* loadParameterMaterial, :593-657 */
  if (!L.find("Nm") || !L.next(&line) || !read_int(line, &iv) || iv < 1) return PTG_ERR_IO;
  m.nmaterial = (int32_t)iv;
  if (!L.next(&line)) return PTG_ERR_IO;  /* "material contents" */
  for (int im = 0; im < m.nmaterial; ++im) {
    if (!L.next(&line)) return PTG_ERR_IO;
    std::vector<std::string> t = tokens(line);
    if (t.empty()) return PTG_ERR_IO;
    b->materials.push_back(t[0]);
    if (!L.next(&line)) return PTG_ERR_IO;  /* a value line */
  }
  auto find_mat = [&](const std::string& name, int upto) {
    for (int i = 0; i < upto && i < (int)b->materials.size(); ++i)
      if (b->materials[i] == name) return i + 1;
    return 0;
  };
  /* loadParameterTransmission, :749-890 */
  if (!L.find("Nt") || !L.next(&line)) return PTG_ERR_IO;
  {
    std::vector<std::string> t = tokens(line);
    long long a, c;
    if (t.size() < 2 || !to_int(t[0], &a) || !to_int(t[1], &c) || a < 1 || c < 1) return PTG_ERR_IO;
    m.nt1 = (int32_t)a;
    m.nt2 = (int32_t)c;
  }
  const size_t tsz = (size_t)(m.nt2 + 1) * m.nt1;
  b->tt_kind.assign(tsz, PTG_TRANS_VALUE);
  b->tt_trans.assign(tsz, 0.0);
  b->tt_spec.assign(tsz, 0.0);
  if (!L.next(&line)) return PTG_ERR_IO;  /* "materials" */
  for (int it = 0; it < m.nt1 * m.nt2; ++it) {
    if (!L.next(&line)) return PTG_ERR_IO;
    std::vector<std::string> t = tokens(line);
    if (t.size() < 4) return PTG_ERR_IO;
    const int i1 = find_mat(t[0], m.nt1), i2 = find_mat(t[1], m.nt2);
    if (!i1 || !i2) return PTG_ERR_IO;
    std::string kt = t[3].substr(0, 5);  /* character(len=5) */
    int kind;
    if (kt == "Value") kind = PTG_TRANS_VALUE;
    else if (kt == "Gamma") kind = PTG_TRANS_GAMMA;
    else if (kt == "TBC") kind = PTG_TRANS_TBC;
    else return PTG_ERR_IO;
    const size_t k = (size_t)(i2 - 1) + (size_t)(m.nt2 + 1) * (i1 - 1);
    b->tt_kind[k] = kind;
    double v2[2];
    if (!L.next(&line) || !read_doubles(line, 2, v2)) return PTG_ERR_IO;
    /* for TBC the first value is the conductance in MW m^-2 K^-1; the caller
       converts it to gamma with ptg_gamma_from_tbc (GammaDeterm, :2499-2599)
       before building the geometry */
    b->tt_trans[k] = kind == PTG_TRANS_TBC ? v2[0] * 1.0e6 : v2[0];
    b->tt_spec[k] = v2[1];
  }
  /* loadGeometry, :894-1171 */
  if (!L.find("Shape") || !L.next(&line)) return PTG_ERR_IO;
  {
    std::vector<std::string> t = tokens(line);
    if (t.empty()) return PTG_ERR_IO;
    if (t[0] == "voronoi") m.kind_grain = PTG_GRAIN_VORONOI;
    else if (t[0] == "bricks") m.kind_grain = PTG_GRAIN_BRICKS;
    else return PTG_ERR_IO;
  }
  if (!L.find("Ng") || !L.next(&line) || !read_int(line, &iv) || iv < 1) return PTG_ERR_IO;
  m.ngrain = (int32_t)iv;
  for (int ig = 0; ig < m.ngrain; ++ig) {
    if (!L.next(&line) || !L.next(&line)) return PTG_ERR_IO;  /* "## grain", "generator" */
    double g3[3];
    if (!L.next(&line) || !read_doubles(line, 3, g3)) return PTG_ERR_IO;
    for (int d = 0; d < 3; ++d) b->grain_generatrix.push_back(g3[d]);
    if (!L.next(&line)) return PTG_ERR_IO;
    std::vector<std::string> t = tokens(line);
    if (t.empty()) return PTG_ERR_IO;
    int shape = PTG_SHAPE_POLYGON;
    double diameter = 0.0;
    if (m.kind_grain == PTG_GRAIN_VORONOI) {
      if (!L.next(&line)) return PTG_ERR_IO;
    } else if (t[0] == "box" || t[0] == "length" || t[0] == "polyhedron") {
      if (!L.next(&line)) return PTG_ERR_IO;
    } else if (t[0] == "sphere" || t[0] == "cylinder") {
      if (!L.next(&line) || !read_doubles(line, 1, &diameter)) return PTG_ERR_IO;
      shape = t[0] == "sphere" ? PTG_SHAPE_SPHERE : PTG_SHAPE_CYLINDER;
    } else {
      return PTG_ERR_IO;
    }
    b->grain_shape.push_back(shape);
    b->grain_diameter.push_back(diameter);
    if (!L.next(&line) || !L.next(&line)) return PTG_ERR_IO;  /* "material", name */
    t = tokens(line);
    if (t.empty()) return PTG_ERR_IO;
    const int im = find_mat(t[0], (int)b->materials.size());
    if (!im) return PTG_ERR_IO;
    b->grain_material.push_back(im);
    long long nsurf = 1;
    if (shape == PTG_SHAPE_POLYGON) {
      if (!L.next(&line) || !L.next(&line)) return PTG_ERR_IO;  /* "# facets", "Nf" */
      if (!L.next(&line) || !read_int(line, &nsurf) || nsurf < 1) return PTG_ERR_IO;
    }
    b->grain_nfacet.push_back((int32_t)nsurf);
    for (long long is = 0; is < nsurf; ++is) {
      if (shape == PTG_SHAPE_POLYGON) {
        if (!L.next(&line) || !L.next(&line)) return PTG_ERR_IO;  /* "# facet", "Nv" */
        long long nv;
        if (!L.next(&line) || !read_int(line, &nv) || nv < 3) return PTG_ERR_IO;
        b->facet_nvertex.push_back((int32_t)nv);
        for (long long k = 0; k < nv; ++k) {
          double v3[3];
          if (!L.next(&line)) return PTG_ERR_IO;  /* "vertex k" */
          if (!L.next(&line) || !read_doubles(line, 3, v3)) return PTG_ERR_IO;
          for (int d = 0; d < 3; ++d) b->facet_vertex.push_back(v3[d]);
        }
      }
      if (!L.next(&line)) return PTG_ERR_IO;
      t = tokens(line);
      if (t.size() < 3) return PTG_ERR_IO;
      int mto;
      if (t[2] == "Internal") mto = PTG_MATERIAL_INTERNAL;
      else {
        const int k = find_mat(t[2], (int)b->materials.size());
        mto = k ? k : PTG_MATERIAL_BOUNDARY;
      }
      b->surf_material_to.push_back(mto);
      if (!L.next(&line)) return PTG_ERR_IO;
      t = tokens(line);
      long long gto;
      if (t.size() < 3 || !to_int(t[2], &gto)) return PTG_ERR_IO;
      b->surf_grain_to.push_back((int32_t)gto);
    }
  }
  m.tt_kind = b->tt_kind.data();
  m.tt_trans = b->tt_trans.data();
  m.tt_spec = b->tt_spec.data();
  m.grain_shape = b->grain_shape.data();
  m.grain_generatrix = b->grain_generatrix.data();
  m.grain_diameter = b->grain_diameter.data();
  m.grain_material = b->grain_material.data();
  m.grain_nfacet = b->grain_nfacet.data();
  m.facet_nvertex = b->facet_nvertex.data();
  m.facet_vertex = b->facet_vertex.data();
  m.surf_material_to = b->surf_material_to.data();
  m.surf_grain_to = b->surf_grain_to.data();
  m.surf_spec = nullptr;
  return PTG_OK;
}

bool read_file(const char* path, Lines* L) {
  std::ifstream f(path);
  if (!f) return false;
  std::string s;
  while (std::getline(f, s)) {
    if (!s.empty() && s.back() == '\r') s.pop_back();
    L->l.push_back(s);
  }
  return true;
}

}  // namespace

struct ptg_anphonbuf {
  ptg_spectrum s;
  std::vector<double> omega, tau, vel, mfp, weight;
};

extern "C" {

int ptg_mcp_load(const char* path, ptg_mcpbuf** out) {
  ptg_mcpbuf* b = nullptr;
  try {
    if (!path || !out) return PTG_ERR_INVALID;
    *out = nullptr;
    Lines L;
    if (!read_file(path, &L)) return PTG_ERR_IO;
    b = ptg::alloc_should_fail() ? nullptr : new (std::nothrow) ptg_mcpbuf();
    if (!b) return PTG_ERR_NOMEM;
    int st = parse_mcp(L, b);
    if (st != PTG_OK) { delete b; return st; }
    *out = b;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    delete b;
    return PTG_ERR_NOMEM;
  } catch (...) {
    delete b;
    return PTG_ERR_INVALID;
  }
}

const ptg_model* ptg_mcpbuf_model(const ptg_mcpbuf* b) { return b ? &b->m : nullptr; }

int ptg_mcpbuf_info(const ptg_mcpbuf* b, int64_t* np, int32_t* nangle, int32_t* kind_mfp,
                    int32_t* nmfp, double* mfp_grid_nm, int32_t* particle_trace, char* material1,
                    int32_t len) {
  if (!b) return PTG_ERR_INVALID;
  if (np) *np = b->np;
  if (nangle) *nangle = b->nangle;
  if (kind_mfp) *kind_mfp = b->kind_mfp;
  if (nmfp) *nmfp = (int32_t)b->mfp_grid.size();
  if (mfp_grid_nm)
    for (size_t i = 0; i < b->mfp_grid.size(); ++i) mfp_grid_nm[i] = b->mfp_grid[i];
  if (particle_trace) *particle_trace = b->particle_trace;
  if (material1 && len > 0) {
    const std::string& s = b->materials.empty() ? std::string() : b->materials[0];
    snprintf(material1, (size_t)len, "%s", s.c_str());
  }
  return PTG_OK;
}

void ptg_mcpbuf_free(ptg_mcpbuf* b) { delete b; }

int ptg_anphon_load(const char* path, ptg_anphonbuf** out) {
  ptg_anphonbuf* b = nullptr;
  try {
    if (!path || !out) return PTG_ERR_INVALID;
    *out = nullptr;
    Lines L;
    if (!read_file(path, &L) || L.l.size() < 7) return PTG_ERR_IO;
    auto value_after = [](const std::string& line, size_t nwords, double* v) {
      std::vector<std::string> t = tokens(line);
      return t.size() > nwords && to_double(t[nwords], v);
    };
    double rtemp, vol, nk, nb;
    if (!value_after(L.l[2], 5, &rtemp) || !value_after(L.l[3], 3, &vol) ||
        !value_after(L.l[4], 4, &nk) || !value_after(L.l[5], 4, &nb) || nk < 1 || nb < 1)
      return PTG_ERR_IO;
    /* one record per (k-point, branch) follows: counts the file cannot hold
       are malformed, not an allocation to attempt */
    if (!(nk <= 2147483647.0) || !(nb <= 2147483647.0) || nk * nb > (double)L.l.size())
      return PTG_ERR_IO;
    b = ptg::alloc_should_fail() ? nullptr : new (std::nothrow) ptg_anphonbuf();
    if (!b) return PTG_ERR_NOMEM;
    const int ik_n = (int)nk, ib_n = (int)nb;
    const size_t n = (size_t)ik_n * ib_n;
    b->omega.resize(n); b->tau.resize(n); b->vel.resize(n); b->mfp.resize(n); b->weight.resize(n);
    size_t li = 7;
    const double conv = 0.03 * (3.14159265358979323846 * 2.0) * 1.0e12;
    for (int ik = 0; ik < ik_n; ++ik) {
      for (int ib = 0; ib < ib_n; ++ib, ++li) {
        if (li >= L.l.size()) { delete b; return PTG_ERR_IO; }
        std::vector<std::string> t = tokens(L.l[li]);
        double v[5];
        if (t.size() < 7) { delete b; return PTG_ERR_IO; }
        for (int k = 0; k < 5; ++k)
          if (!to_double(t[2 + k], &v[k])) { delete b; return PTG_ERR_IO; }
        const size_t m = (size_t)ib + (size_t)ib_n * ik;
        b->omega[m] = v[0] * conv;
        b->tau[m] = v[1];
        b->vel[m] = v[2];
        b->mfp[m] = v[3];
        b->weight[m] = v[4];
      }
    }
    ptg_spectrum& s = b->s;
    s.nbranch = ib_n;
    s.nkpoint = ik_n;
    s.rtemp = rtemp;
    s.vol = vol;
    s.omega = b->omega.data();
    s.tau = b->tau.data();
    s.vel = b->vel.data();
    s.mfp = b->mfp.data();
    s.weight = b->weight.data();
    *out = b;
    return PTG_OK;
  } catch (const std::bad_alloc&) {
    delete b;
    return PTG_ERR_NOMEM;
  } catch (...) {
    delete b;
    return PTG_ERR_INVALID;
  }
}

const ptg_spectrum* ptg_anphonbuf_spectrum(const ptg_anphonbuf* b) { return b ? &b->s : nullptr; }

void ptg_anphonbuf_free(ptg_anphonbuf* b) { delete b; }

int ptg_anphon_write(const char* path, const ptg_spectrum* s) {
  if (!path || !s || s->nbranch < 1 || s->nkpoint < 1) return PTG_ERR_INVALID;
  FILE* f = fopen(path, "w");
  if (!f) return PTG_ERR_IO;
  const double conv = 0.03 * (3.14159265358979323846 * 2.0) * 1.0e12;
  fprintf(f, "# anphon mode table\n# columns: ik ib omega[cm^-1] tau[ps] vel[m s^-1] MFP weight\n");
  fprintf(f, "# reference temperature K = %.17g\n", s->rtemp);
  fprintf(f, "# vol = %.17g\n", s->vol);
  fprintf(f, "# nkpoint total = %d\n", s->nkpoint);
  fprintf(f, "# nbranch total = %d\n", s->nbranch);
  fprintf(f, "# ik ib omega tau vel MFP weight\n");
  for (int ik = 0; ik < s->nkpoint; ++ik) {
    for (int ib = 0; ib < s->nbranch; ++ib) {
      const size_t m = (size_t)ib + (size_t)s->nbranch * ik;
      fprintf(f, "%d %d %.17g %.17g %.17g %.17g %.17g\n", ik + 1, ib + 1, s->omega[m] / conv,
              s->tau[m], s->vel[m], s->mfp ? s->mfp[m] : 0.0, s->weight[m]);
    }
  }
  return fclose(f) == 0 ? PTG_OK : PTG_ERR_IO;
}

}  // extern "C"
