/*
 * ptrans_oracle.cpp - TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the P-TRANS Monte Carlo ray-tracing hot path
 * (Fortran module RTMC, src/RTMCphon.f90), kept close to the reference's own
 * structure: grains of surfaces, a linear scan of the box grain plus the
 * current grain per free flight, the reference's intersection, reflection and
 * transmission rules, the reference's 1e-7 nm nudge and out-of-box check,
 * Simpson's rule over the incident angle and the kappa sum of fileoutput.
 *
 * It differs from the reference only where the reference cannot be
 * reproduced or is undefined:
 *   - random numbers come from Philox4x32-10 with the counter layout of
 *     include/ptrans_gpu.h instead of the clock-seeded gfortran generator
 *     (src/RTMCphon.f90:3314-3330);
 *   - log and sin/cos of 2*pi*u use oracle_math.h so that a device
 *     restatement can replay trajectories bit for bit;
 *   - a phonon in grain 0 (box) only scans grain 0; the reference's
 *     "do ig=0,whichV,whichV" has a zero step there (src/RTMCphon.f90:2012);
 *   - quantities the reference leaves uninitialised (EMFP when the bulk MFP
 *     equals the last grid point, src/RTMCphon.f90:2729-2743; the radius of
 *     polygon surfaces; the start grain when no grain is incident) get the
 *     values documented at their use.
 * Parity status: PARITY UNPINNED (see ptrans_oracle.h).
 *
 * Used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
 */
#include "ptrans_oracle.h"
#include "oracle_math.h"

#include <omp.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

namespace {

const double M_PI_D = 3.14159265358979323846;
const double M_PI_2_D = M_PI_D * 0.5;
const double HBAR = 1.054571e-34;     /* src/RTMCphon.f90:65 */
const double KB = 1.3806503e-23;      /* src/RTMCphon.f90:66 */
const double SMALL_VAL = 1.0e-5;      /* src/RTMCphon.f90:67 */
const double BALLISTIC = 1.0e10;      /* src/RTMCphon.f90:1686 */

struct Surf {
  int incident = 0, internal = 1, grain_inside = 0, grain_outside = 0, nvertex = 0;
  std::vector<double> vertex;          /* 3*(nvertex+1): vertex(:,k) at 3*k */
  double normal[3] = {0, 0, 0};
  double tangent[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  /* tangent(:,j) at 3*j */
  double radius = 0, center[3] = {0, 0, 0};
  int shape = PTG_SHAPE_POLYGON, kind_trans = PTG_TRANS_VALUE, mat1 = 0, mat2 = 0;
  double spec = 0, tparam = 0;
};

struct Grain {
  int incident = 0;
  double gen[3] = {0, 0, 0};
  std::vector<Surf> s;
};

}  // namespace

struct orc_handle {
  double box[3] = {0, 0, 0}, scope[2] = {1, 1};
  int face_kind[6] = {0, 0, 0, 0, 0, 0};
  int kind_grain = PTG_GRAIN_VORONOI, ngrain = 0, igrain_fill = -1, nmaterial = 1;
  std::vector<Grain> g;
  /* spectrum */
  int nb = 1, nk = 1;
  double rtemp = 300, vol = 1, max_omega = 1;
  std::vector<double> omega, tau, vel, mfp, weight;
};

namespace {

inline double dot3(const double* a, const double* b) {
  /* gfortran dot_product order: ((a1*b1 + a2*b2) + a3*b3) */
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
inline void cross3(const double* a, const double* b, double* c) {
  /* cross_product, src/RTMCphon.f90:185-192 */
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* setupSurfaceGeometry, src/RTMCphon.f90:1433-1491 */
void setup_surface_geometry(Surf& s) {
  if (s.shape != PTG_SHAPE_POLYGON) return;
  int n = s.nvertex;
  const double* v = s.vertex.data();
  for (int d = 0; d < 3; ++d) s.center[d] = 0.0;
  for (int iv = 0; iv < n; ++iv)
    for (int d = 0; d < 3; ++d) s.center[d] = s.center[d] + v[3 * iv + d];
  for (int d = 0; d < 3; ++d) s.center[d] = 1.0 / n * s.center[d];
  double nrm[3] = {0, 0, 0};
  double a[3], b[3], c[3];
  for (int iv = 0; iv < n - 1; ++iv) {
    for (int d = 0; d < 3; ++d) {
      a[d] = v[3 * (iv + 1) + d] - v[3 * iv + d];
      b[d] = v[3 * (iv + 2) + d] - v[3 * iv + d];
    }
    cross3(a, b, c);
    double len = sqrt(dot3(c, c));
    for (int d = 0; d < 3; ++d) nrm[d] = nrm[d] + c[d] / len;
  }
  for (int d = 0; d < 3; ++d) {
    a[d] = v[3 * n + d] - v[3 * (n - 1) + d];
    b[d] = v[3 * 1 + d] - v[3 * (n - 1) + d];
  }
  cross3(a, b, c);
  double len = sqrt(dot3(c, c));
  for (int d = 0; d < 3; ++d) nrm[d] = nrm[d] + c[d] / len;
  for (int d = 0; d < 3; ++d) s.normal[d] = 1.0 / n * nrm[d];
  double* t = s.tangent;
  for (int d = 0; d < 3; ++d) t[6 + d] = s.normal[d];
  const double* N = s.normal;
  if (fabs(N[2]) == 1.0 || (N[0] * N[0] == 0.0 && N[1] * N[1] == 0.0)) {
    t[3] = 0; t[4] = 1; t[5] = 0;
    t[0] = 1; t[1] = 0; t[2] = 0;
  } else {
    double q = sqrt(N[0] * N[0] + N[1] * N[1]);
    t[3] = -N[1] / q; t[4] = N[0] / q; t[5] = 0.0;
    cross3(&t[3], &t[6], &t[0]);
  }
}

double tt_get(const double* arr, const ptg_model* m, int imat2, int imat1) {
  /* param%X(imat2, imat1), allocated (nt2+1, nt1) */
  return arr[(imat2 - 1) + (m->nt2 + 1) * (imat1 - 1)];
}
int tt_geti(const int32_t* arr, const ptg_model* m, int imat2, int imat1) {
  return arr[(imat2 - 1) + (m->nt2 + 1) * (imat1 - 1)];
}

/* Gaussian from 12 uniforms (normal_distribution, src/RTMCphon.f90:1188-1199);
   the uniforms come from Philox keyed by fluct_seed, counter
   (j, 0x464C, surface, 0), j = 0..2, each word w -> (w + 0.5) * 2^-32. */
double fluct_normal(uint64_t seed, int surf, double mean, double dev) {
  double sum = 0.0;
  for (uint32_t j = 0; j < 3; ++j) {
    orc::Philox4 p = orc::philox4x32_10(j, 0x464Cu, (uint32_t)surf, 0u, (uint32_t)seed,
                                        (uint32_t)(seed >> 32));
    for (int w = 0; w < 4; ++w) sum = sum + ((double)p.v[w] + 0.5) * (1.0 / 4294967296.0);
  }
  return (sum - 6.0) * dev + mean;
}

int check_tt(const ptg_model* m, int imat2, int imat1) {
  return imat2 >= 1 && imat2 <= m->nt2 + 1 && imat1 >= 1 && imat1 <= m->nt1;
}

}  // namespace

extern "C" {

int orc_build_model(const ptg_model* m, const ptg_spectrum* sp, orc_handle** out) {
  if (!m || !out) return PTG_ERR_INVALID;
  *out = nullptr;
  if (m->ngrain < 1 || (m->kind_grain != PTG_GRAIN_VORONOI && m->kind_grain != PTG_GRAIN_BRICKS))
    return PTG_ERR_INVALID;
  orc_handle* h = new orc_handle();
  for (int d = 0; d < 3; ++d) h->box[d] = m->box[d];
  h->scope[0] = m->scope[0];
  h->scope[1] = m->scope[1];
  for (int f = 0; f < 6; ++f) h->face_kind[f] = m->face_kind[f];
  h->kind_grain = m->kind_grain;
  h->ngrain = m->ngrain;
  h->nmaterial = m->nmaterial;
  h->igrain_fill = (m->kind_grain == PTG_GRAIN_BRICKS) ? m->ngrain + 1 : -1;
  h->g.resize(m->ngrain + 1 + (m->kind_grain == PTG_GRAIN_BRICKS ? 1 : 0));
  if (sp) {
    h->nb = sp->nbranch; h->nk = sp->nkpoint;
    size_t n = (size_t)h->nb * h->nk;
    h->omega.assign(sp->omega, sp->omega + n);
    h->tau.assign(sp->tau, sp->tau + n);
    h->vel.assign(sp->vel, sp->vel + n);
    h->weight.assign(sp->weight, sp->weight + n);
    if (sp->mfp) h->mfp.assign(sp->mfp, sp->mfp + n); else h->mfp.assign(n, 0.0);
    h->rtemp = sp->rtemp; h->vol = sp->vol;
    double mx = h->omega[0];
    for (size_t i = 1; i < n; ++i) if (h->omega[i] > mx) mx = h->omega[i];
    h->max_omega = mx;
  }
  const double X = m->box[0], Y = m->box[1], Z = m->box[2];
  /* setupBoxGrain, src/RTMCphon.f90:1253-1332 (final vertex orders) */
  {
    Grain& box = h->g[0];
    box.incident = 0;
    const double V[6][4][3] = {
        {{0, 0, 0}, {0, 0, Z}, {0, Y, Z}, {0, Y, 0}},
        {{X, 0, 0}, {X, Y, 0}, {X, Y, Z}, {X, 0, Z}},
        {{0, 0, 0}, {X, 0, 0}, {X, 0, Z}, {0, 0, Z}},
        {{X, Y, 0}, {0, Y, 0}, {0, Y, Z}, {X, Y, Z}},
        {{0, 0, 0}, {0, Y, 0}, {X, Y, 0}, {X, 0, 0}},
        {{0, Y, Z}, {0, 0, Z}, {X, 0, Z}, {X, Y, Z}}};
    box.s.resize(6);
    for (int f = 0; f < 6; ++f) {
      Surf& s = box.s[f];
      s.incident = 0; s.internal = 1; s.grain_inside = 0; s.grain_outside = 0;
      s.shape = PTG_SHAPE_POLYGON;
      s.radius = 0.0;
      s.nvertex = 4;
      s.vertex.resize(15);
      for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 3; ++d) s.vertex[3 * k + d] = V[f][k][d];
      for (int d = 0; d < 3; ++d) s.vertex[12 + d] = V[f][0][d];
      setup_surface_geometry(s);
      s.spec = m->cellspec[f];
      s.kind_trans = PTG_TRANS_VALUE;
      s.tparam = 0.0;
    }
  }
  /* grains, src/RTMCphon.f90:968-1171 */
  int fpos = 0, vpos = 0, spos = 0;
  int gsurf_index = 6;  /* built-surface index used to key the fluctuation */
  for (int ig = 1; ig <= m->ngrain; ++ig) {
    Grain& gr = h->g[ig];
    gr.incident = 0;
    for (int d = 0; d < 3; ++d) gr.gen[d] = m->grain_generatrix[3 * (ig - 1) + d];
    int shape = (m->kind_grain == PTG_GRAIN_VORONOI) ? PTG_SHAPE_POLYGON : m->grain_shape[ig - 1];
    double diameter = (shape == PTG_SHAPE_POLYGON) ? 0.0 : m->grain_diameter[ig - 1];
    int imat1 = m->grain_material[ig - 1];
    if (imat1 < 1 || imat1 > m->nmaterial) { orc_free(h); return PTG_ERR_INVALID; }
    int ns = (shape == PTG_SHAPE_POLYGON) ? m->grain_nfacet[ig - 1] : 1;
    gr.s.resize(ns);
    for (int is = 0; is < ns; ++is, ++spos, ++gsurf_index) {
      Surf& s = gr.s[is];
      s.incident = 0; s.internal = 1; s.grain_inside = ig; s.mat1 = imat1; s.shape = shape;
      for (int d = 0; d < 3; ++d) s.center[d] = gr.gen[d];
      s.radius = diameter * 0.5;
      if (shape == PTG_SHAPE_POLYGON) {
        int nv = m->facet_nvertex[fpos++];
        if (nv < 3) { orc_free(h); return PTG_ERR_INVALID; }
        s.nvertex = nv;
        s.vertex.resize(3 * (nv + 1));
        for (int k = 0; k < nv; ++k)
          for (int d = 0; d < 3; ++d) s.vertex[3 * k + d] = m->facet_vertex[3 * (vpos + k) + d];
        for (int d = 0; d < 3; ++d) s.vertex[3 * nv + d] = s.vertex[d];
        vpos += nv;
        setup_surface_geometry(s);
        /* isIncidentSurface / isInternalSurface, src/RTMCphon.f90:1202-1246 */
        bool all_xle0 = true, all_xgeX = true, all_yle0 = true, all_ygeY = true,
             all_zle0 = true, all_zgeZ = true;
        for (int k = 0; k <= nv; ++k) {
          const double* p = &s.vertex[3 * k];
          if (!(p[0] <= 0.0)) all_xle0 = false;
          if (!(p[0] >= X)) all_xgeX = false;
          if (!(p[1] <= 0.0)) all_yle0 = false;
          if (!(p[1] >= Y)) all_ygeY = false;
          if (!(p[2] <= 0.0)) all_zle0 = false;
          if (!(p[2] >= Z)) all_zgeZ = false;
        }
        if (all_xle0) { gr.incident = 1; s.incident = 1; s.internal = 0; }
        if (all_xle0 || all_xgeX || all_yle0 || all_ygeY || all_zle0 || all_zgeZ) s.internal = 0;
      } else if (shape == PTG_SHAPE_CAPPED) {
        /* extension: capped cylinder, axis end points c -/+ axis/2 (closed) */
        if (!m->grain_axis) { orc_free(h); return PTG_ERR_INVALID; }
        const double* ax = m->grain_axis + 3 * (ig - 1);
        s.nvertex = 2;
        s.vertex.resize(9);
        for (int d = 0; d < 3; ++d) {
          s.vertex[d] = s.center[d] - 0.5 * ax[d];
          s.vertex[3 + d] = s.center[d] + 0.5 * ax[d];
          s.vertex[6 + d] = s.vertex[d];
        }
      } else {
        s.nvertex = 0;
      }
      int mto = m->surf_material_to[spos];
      s.grain_outside = m->surf_grain_to[spos];
      if (!s.internal) continue;
      if (mto == PTG_MATERIAL_INTERNAL) {
        s.mat2 = 1;
        s.grain_outside = h->igrain_fill;
      } else {
        if (mto < 1 || mto > m->nmaterial) { orc_free(h); return PTG_ERR_INVALID; }
        s.mat2 = mto;
      }
      if (!check_tt(m, s.mat2, s.mat1)) { orc_free(h); return PTG_ERR_INVALID; }
      s.spec = tt_get(m->tt_spec, m, s.mat2, s.mat1);
      if (m->specfluc > 0.0) {
        s.spec = fluct_normal(m->fluct_seed, gsurf_index, s.spec, m->specfluc);
        if (s.spec < 0.0) s.spec = 0.0;
        if (s.spec > 1.0) s.spec = 1.0;
      }
      if (m->surf_spec) s.spec = m->surf_spec[spos];
      s.kind_trans = tt_geti(m->tt_kind, m, s.mat2, s.mat1);
      s.tparam = tt_get(m->tt_trans, m, s.mat2, s.mat1);
    }
  }
  /* setupFillGrain, src/RTMCphon.f90:1336-1398 */
  if (m->kind_grain == PTG_GRAIN_BRICKS) {
    Grain& fill = h->g[h->igrain_fill];
    fill.incident = 0;
    int sp2 = 0;
    for (int ig = 1; ig <= m->ngrain; ++ig) {
      for (size_t js = 0; js < h->g[ig].s.size(); ++js, ++sp2) {
        const Surf& sj = h->g[ig].s[js];
        if (!sj.internal) continue;
        Surf s;
        s.incident = 0; s.internal = 1; s.grain_inside = h->igrain_fill;
        s.mat1 = 1; s.mat2 = sj.mat1; s.shape = sj.shape;
        for (int d = 0; d < 3; ++d) s.center[d] = sj.center[d];
        s.radius = sj.radius;
        s.nvertex = sj.nvertex;
        if (s.nvertex > 0) {
          int n = s.nvertex;
          s.vertex.resize(3 * (n + 1));
          for (int iv = 0; iv <= n; ++iv)
            for (int d = 0; d < 3; ++d) s.vertex[3 * iv + d] = sj.vertex[3 * (n - iv) + d];
        }
        setup_surface_geometry(s);
        s.grain_outside = sj.grain_inside;
        if (!check_tt(m, s.mat2, s.mat1)) { orc_free(h); return PTG_ERR_INVALID; }
        s.spec = tt_get(m->tt_spec, m, s.mat2, s.mat1);
        if (m->surf_spec) s.spec = m->surf_spec[sp2];
        s.kind_trans = tt_geti(m->tt_kind, m, s.mat2, s.mat1);
        s.tparam = tt_get(m->tt_trans, m, s.mat2, s.mat1);
        fill.s.push_back(s);
      }
    }
  }
  *out = h;
  return PTG_OK;
}

int orc_from_geometry(const ptg_geometry* G, const ptg_spectrum* sp, orc_handle** out) {
  if (!G || !out) return PTG_ERR_INVALID;
  orc_handle* h = new orc_handle();
  for (int d = 0; d < 3; ++d) h->box[d] = G->box[d];
  h->scope[0] = G->scope[0]; h->scope[1] = G->scope[1];
  for (int f = 0; f < 6; ++f) h->face_kind[f] = G->face_kind[f];
  h->kind_grain = G->kind_grain; h->ngrain = G->ngrain; h->igrain_fill = G->igrain_fill;
  h->nmaterial = G->nmaterial;
  h->g.resize(G->ngrain_total);
  for (int ig = 0; ig < G->ngrain_total; ++ig) {
    Grain& gr = h->g[ig];
    gr.incident = G->grain_incident[ig];
    for (int d = 0; d < 3; ++d) gr.gen[d] = G->grain_generatrix[3 * ig + d];
    for (int k = G->grain_begin[ig]; k < G->grain_begin[ig + 1]; ++k) {
      Surf s;
      s.shape = G->shape[k]; s.nvertex = G->nvertex[k];
      if (s.nvertex > 0) {
        s.vertex.assign(G->vertex + 3 * (size_t)G->vertex_begin[k],
                        G->vertex + 3 * ((size_t)G->vertex_begin[k] + s.nvertex + 1));
      }
      for (int d = 0; d < 3; ++d) { s.normal[d] = G->normal[3 * k + d]; s.center[d] = G->center[3 * k + d]; }
      for (int d = 0; d < 9; ++d) s.tangent[d] = G->tangent[9 * k + d];
      s.radius = G->radius[k]; s.kind_trans = G->kind_trans[k]; s.spec = G->specularity[k];
      s.tparam = G->trans_param[k]; s.grain_inside = G->grain_inside[k];
      s.grain_outside = G->grain_outside[k]; s.internal = G->internal[k];
      s.incident = G->incident[k]; s.mat1 = G->material1[k]; s.mat2 = G->material2[k];
      gr.s.push_back(s);
    }
  }
  if (sp) {
    h->nb = sp->nbranch; h->nk = sp->nkpoint;
    size_t n = (size_t)h->nb * h->nk;
    h->omega.assign(sp->omega, sp->omega + n);
    h->tau.assign(sp->tau, sp->tau + n);
    h->vel.assign(sp->vel, sp->vel + n);
    h->weight.assign(sp->weight, sp->weight + n);
    if (sp->mfp) h->mfp.assign(sp->mfp, sp->mfp + n); else h->mfp.assign(n, 0.0);
    h->rtemp = sp->rtemp; h->vol = sp->vol;
    double mx = h->omega[0];
    for (size_t i = 1; i < n; ++i) if (h->omega[i] > mx) mx = h->omega[i];
    h->max_omega = mx;
  }
  *out = h;
  return PTG_OK;
}

void orc_free(orc_handle* h) { delete h; }

int orc_geometry_sizes(const orc_handle* h, int32_t* ngt, int32_t* ns, int32_t* nvt) {
  if (!h) return PTG_ERR_INVALID;
  int s = 0, v = 0;
  for (const Grain& g : h->g)
    for (const Surf& x : g.s) { ++s; v += x.nvertex > 0 ? x.nvertex + 1 : 0; }
  if (ngt) *ngt = (int32_t)h->g.size();
  if (ns) *ns = s;
  if (nvt) *nvt = v;
  return PTG_OK;
}

int orc_geometry_export(const orc_handle* h, int32_t* grain_begin, int32_t* grain_incident,
                        double* grain_generatrix, int32_t* shape, int32_t* nvertex,
                        int32_t* vertex_begin, double* vertex, double* normal, double* tangent,
                        double* center, double* radius, int32_t* kind_trans, double* specularity,
                        double* trans_param, int32_t* grain_inside, int32_t* grain_outside,
                        int32_t* internal, int32_t* incident, int32_t* material1,
                        int32_t* material2) {
  if (!h) return PTG_ERR_INVALID;
  int k = 0, v = 0;
  for (size_t ig = 0; ig < h->g.size(); ++ig) {
    const Grain& g = h->g[ig];
    grain_begin[ig] = k;
    grain_incident[ig] = g.incident;
    for (int d = 0; d < 3; ++d) grain_generatrix[3 * ig + d] = g.gen[d];
    for (const Surf& s : g.s) {
      shape[k] = s.shape; nvertex[k] = s.nvertex; vertex_begin[k] = v;
      if (s.nvertex > 0) {
        for (int i = 0; i < 3 * (s.nvertex + 1); ++i) vertex[3 * v + i] = s.vertex[i];
        v += s.nvertex + 1;
      }
      for (int d = 0; d < 3; ++d) { normal[3 * k + d] = s.normal[d]; center[3 * k + d] = s.center[d]; }
      for (int d = 0; d < 9; ++d) tangent[9 * k + d] = s.tangent[d];
      radius[k] = s.radius; kind_trans[k] = s.kind_trans; specularity[k] = s.spec;
      trans_param[k] = s.tparam; grain_inside[k] = s.grain_inside;
      grain_outside[k] = s.grain_outside; internal[k] = s.internal; incident[k] = s.incident;
      material1[k] = s.mat1; material2[k] = s.mat2;
      ++k;
    }
  }
  grain_begin[h->g.size()] = k;
  return PTG_OK;
}

}  // extern "C"

/* ------------------------------------------------------------------------ */
/* transport                                                                */
/* ------------------------------------------------------------------------ */
namespace {

struct Task {
  double lambda;        /* gray MFP [nm]; 1e10 = ballistic */
  double cth, sth;      /* cos / sin of the incident polar angle */
  int ib, ik;
  double omega;         /* mode frequency (Gamma/TBC threshold) */
};

struct Rng {
  uint32_t k0, k1, c1, slo, shi;
  void block(uint32_t flight, uint32_t sub, double* d0, double* d1) const {
    orc::Philox4 p = orc::philox4x32_10(flight, sub | c1, slo, shi, k0, k1);
    *d0 = orc::u52(p.v[0], p.v[1]);
    *d1 = orc::u52(p.v[2], p.v[3]);
  }
};

/* calcSurfaceDistancePolygon, src/RTMCphon.f90:2907-2959 */
bool dist_polygon(const double* R0, const double* D, const Surf& s, double* L) {
  double cosangle = dot3(D, s.normal);
  if (cosangle <= 0.0) return false;
  double w[3];
  for (int d = 0; d < 3; ++d) w[d] = s.vertex[d] - R0[d];
  double Lh = dot3(w, s.normal) / cosangle;
  if (Lh < 0.0) return false;
  double Rh[3];
  for (int d = 0; d < 3; ++d) Rh[d] = R0[d] + D[d] * Lh;
  double c1[3], ci[3], Ra[3], Rb[3];
  for (int i = 0; i < s.nvertex; ++i) {
    for (int d = 0; d < 3; ++d) {
      Ra[d] = s.vertex[3 * (i + 1) + d] - s.vertex[3 * i + d];
      Rb[d] = Rh[d] - s.vertex[3 * i + d];
    }
    cross3(Ra, Rb, ci);
    if (i == 0) {
      for (int d = 0; d < 3; ++d) c1[d] = ci[d];
    } else if (dot3(c1, ci) < 0.0) {
      return false;
    }
  }
  *L = Lh;
  return true;
}

/* isInsidePolygon, src/RTMCphon.f90:2961-2983 */
bool inside_polygon(const Surf& s, const double* Rh) {
  double c1[3], ci[3], Ra[3], Rb[3];
  for (int i = 0; i < s.nvertex; ++i) {
    for (int d = 0; d < 3; ++d) {
      Ra[d] = s.vertex[3 * (i + 1) + d] - s.vertex[3 * i + d];
      Rb[d] = Rh[d] - s.vertex[3 * i + d];
    }
    cross3(Ra, Rb, ci);
    if (i == 0) {
      for (int d = 0; d < 3; ++d) c1[d] = ci[d];
    } else if (dot3(c1, ci) < 0.0) {
      return false;
    }
  }
  return true;
}

/* calcSurfaceDistanceSphere, src/RTMCphon.f90:2985-3038 */
bool dist_sphere(const double* R0, const double* D, const Surf& s, double* L) {
  double Rsc[3];
  for (int d = 0; d < 3; ++d) Rsc[d] = s.center[d] - R0[d];
  double RD = dot3(Rsc, D);
  double RR = dot3(Rsc, Rsc);
  double r2 = s.radius * s.radius;
  if (RR > r2 - 1e-10) {
    if (RD <= 0.0) return false;
  }
  double Dd = RD * RD + r2 - RR;
  if (Dd < 0.0) return false;
  double sq = sqrt(Dd);
  double L1 = RD - sq, L2 = RD + sq;
  if (L1 > 0.0) *L = L1;
  else if (L2 > 0.0) *L = L2;
  else return false;
  return true;
}

/* calcSurfaceDistanceCylinder, src/RTMCphon.f90:3040-3088 */
bool dist_cylinder(const double* R0, const double* D, const Surf& s, double boxz, double* L) {
  double Rsc0 = s.center[0] - R0[0], Rsc1 = s.center[1] - R0[1];
  double t0 = D[0], t1 = D[1];
  double nv = t0 * t0 + t1 * t1 + 0.0 * 0.0;
  double sq_nv = sqrt(nv);
  t0 = t0 / sq_nv;
  t1 = t1 / sq_nv;
  double RD = Rsc0 * t0 + Rsc1 * t1;
  double RR = Rsc0 * Rsc0 + Rsc1 * Rsc1;
  double r2 = s.radius * s.radius;
  double Dd = RD * RD + r2 - RR;
  if (Dd < 0.0) return false;
  double sq = sqrt(Dd);
  double L1 = RD - sq, L2 = RD + sq;
  double Lh;
  if (L1 > 0.0) Lh = L1;
  else if (L2 > 0.0) Lh = L2;
  else return false;
  Lh = Lh / sqrt(D[0] * D[0] + D[1] * D[1]);
  double z = R0[2] + D[2] * Lh;
  if (z < 0.0 || boxz < z) return false;
  *L = Lh;
  return true;
}

/* Axis of a capped cylinder from its end points A (vertex 0) and B
   (vertex 1): unit axis a, half length hl. */
void capped_axis(const Surf& s, double* a, double* hl) {
  double e[3];
  for (int d = 0; d < 3; ++d) e[d] = s.vertex[3 + d] - s.vertex[d];
  const double len = sqrt(dot3(e, e));
  for (int d = 0; d < 3; ++d) a[d] = e[d] / len;
  *hl = 0.5 * len;
}

/* Extension: ray against a capped cylinder (centre c, unit axis a, radius r,
   half length hl), written like the reference's quadric tests: the nearest
   strictly positive distance over the lateral surface (axial coordinate
   within the caps) and the two cap discs (radial distance within r). */
bool dist_capped(const double* R0, const double* D, const Surf& s, double* L) {
  double a[3], hl;
  capped_axis(s, a, &hl);
  double w[3];
  for (int d = 0; d < 3; ++d) w[d] = R0[d] - s.center[d];
  const double s0 = dot3(w, a), ds = dot3(D, a);
  double wp[3], dp[3];
  for (int d = 0; d < 3; ++d) {
    wp[d] = w[d] - s0 * a[d];
    dp[d] = D[d] - ds * a[d];
  }
  const double r2 = s.radius * s.radius;
  double best = 0.0;
  bool hit = false;
  const double A2 = dot3(dp, dp);
  if (A2 > 0.0) {
    const double B = dot3(wp, dp), C = dot3(wp, wp) - r2;
    const double disc = B * B - A2 * C;
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

/* Outward normal of the capped-cylinder piece nearest to R: a cap (+-a) when
   the axial distance to it is smaller than the radial distance to the
   mantle, else the radial direction. */
void capped_normal(const Surf& s, const double* R, double* N) {
  double a[3], hl;
  capped_axis(s, a, &hl);
  double w[3];
  for (int d = 0; d < 3; ++d) w[d] = R[d] - s.center[d];
  const double sa = dot3(w, a);
  double wp[3];
  for (int d = 0; d < 3; ++d) wp[d] = w[d] - sa * a[d];
  const double rho = sqrt(dot3(wp, wp));
  if (fabs(fabs(sa) - hl) < fabs(rho - s.radius)) {
    const double sg = (sa < 0.0) ? -1.0 : 1.0;
    for (int d = 0; d < 3; ++d) N[d] = sg * a[d];
  } else {
    for (int d = 0; d < 3; ++d) N[d] = wp[d] / rho;
  }
}

bool surface_distance(const orc_handle* h, const double* R0, const double* D, const Surf& s,
                      double* L) {
  switch (s.shape) {
    case PTG_SHAPE_POLYGON: return dist_polygon(R0, D, s, L);
    case PTG_SHAPE_SPHERE: return dist_sphere(R0, D, s, L);
    case PTG_SHAPE_CYLINDER: return dist_cylinder(R0, D, s, h->box[2], L);
    case PTG_SHAPE_CAPPED: return dist_capped(R0, D, s, L);
  }
  return false;
}

/* calcSurfaceNormal*, src/RTMCphon.f90:3119-3179 */
void surface_normal(const Surf& s, const double* R, double* N) {
  if (s.shape == PTG_SHAPE_POLYGON) {
    for (int d = 0; d < 3; ++d) N[d] = s.normal[d];
    return;
  }
  if (s.shape == PTG_SHAPE_CAPPED) {
    capped_normal(s, R, N);
    return;
  }
  double Rcs[3];
  if (s.shape == PTG_SHAPE_SPHERE) {
    for (int d = 0; d < 3; ++d) Rcs[d] = R[d] - s.center[d];
  } else {
    Rcs[2] = 0.0;
    Rcs[0] = R[0] - s.center[0];
    Rcs[1] = R[1] - s.center[1];
  }
  double rr = dot3(Rcs, Rcs);
  double inv = 1.0 / sqrt(rr);
  for (int d = 0; d < 3; ++d) N[d] = Rcs[d] * inv;
  if (rr > s.radius * s.radius)
    for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
}

/* calcSurfaceRotation*, src/RTMCphon.f90:3181-3301; Rm col-major */
void surface_rotation(const Surf& s, const double* R, double* Rm) {
  if (s.shape == PTG_SHAPE_POLYGON) {
    for (int d = 0; d < 9; ++d) Rm[d] = s.tangent[d];
    return;
  }
  double n[3];
  if (s.shape == PTG_SHAPE_CAPPED) {
    /* frame around the piece's normal, built like the sphere's */
    capped_normal(s, R, n);
    for (int d = 0; d < 3; ++d) Rm[6 + d] = n[d];
    if (fabs(n[2]) == 1.0 || (n[0] * n[0] == 0.0 && n[1] * n[1] == 0.0)) {
      Rm[3] = 0; Rm[4] = 1; Rm[5] = 0; Rm[0] = 1; Rm[1] = 0; Rm[2] = 0;
    } else {
      double q = sqrt(n[0] * n[0] + n[1] * n[1]);
      Rm[3] = -n[1] / q; Rm[4] = n[0] / q; Rm[5] = 0.0;
      cross3(&Rm[3], &Rm[6], &Rm[0]);
    }
  } else if (s.shape == PTG_SHAPE_SPHERE) {
    double Rcs[3];
    for (int d = 0; d < 3; ++d) Rcs[d] = R[d] - s.center[d];
    double inv = 1.0 / sqrt(dot3(Rcs, Rcs));
    for (int d = 0; d < 3; ++d) n[d] = Rcs[d] * inv;
    for (int d = 0; d < 3; ++d) Rm[6 + d] = n[d];
    if (fabs(n[2]) == 1.0 || (n[0] * n[0] == 0.0 && n[1] * n[1] == 0.0)) {
      Rm[3] = 0; Rm[4] = 1; Rm[5] = 0; Rm[0] = 1; Rm[1] = 0; Rm[2] = 0;
    } else {
      double q = sqrt(n[0] * n[0] + n[1] * n[1]);
      Rm[3] = -n[1] / q; Rm[4] = n[0] / q; Rm[5] = 0.0;
      cross3(&Rm[3], &Rm[6], &Rm[0]);
    }
  } else {
    double Nn[3];
    Nn[0] = R[0] - s.center[0];
    Nn[1] = R[1] - s.center[1];
    Nn[2] = 0.0;
    double inv = 1.0 / sqrt(dot3(Nn, Nn));
    for (int d = 0; d < 3; ++d) Nn[d] = Nn[d] * inv;
    for (int d = 0; d < 3; ++d) Rm[6 + d] = Nn[d];
    if (fabs(Nn[0]) == 1.0 || (Nn[0] * Nn[0] == 0.0 && Nn[1] * Nn[1] == 0.0)) {
      Rm[3] = 0; Rm[4] = 1; Rm[5] = 0; Rm[0] = 1; Rm[1] = 0; Rm[2] = 0;
    } else {
      double q = sqrt(Nn[0] * Nn[0] + Nn[1] * Nn[1]);
      Rm[3] = -Nn[1] / q; Rm[4] = Nn[0] / q; Rm[5] = 0.0;
      cross3(&Rm[3], &Rm[6], &Rm[0]);
    }
  }
}

/* determinTransmit threshold, src/RTMCphon.f90:2384-2413.  omega_draw is
   only read for several materials with Gamma/TBC. */
double transmit_threshold(const orc_handle* h, const Surf& s, const Task& t, double omega_draw) {
  switch (s.kind_trans) {
    case PTG_TRANS_VALUE: return s.tparam;
    case PTG_TRANS_GAMMA:
    case PTG_TRANS_TBC:
      if (h->nmaterial == 1) {
        return 1.0 / (s.tparam * t.omega / h->max_omega + 1.0);
      } else {
        double t11 = 1.0 / (s.tparam + 1.0);
        return t11 + omega_draw * (1 - t11);
      }
  }
  return 0.0;
}

bool needs_omega_draw(const orc_handle* h, const Surf& s) {
  return h->nmaterial != 1 &&
         (s.kind_trans == PTG_TRANS_GAMMA || s.kind_trans == PTG_TRANS_TBC);
}

inline const Surf& surf_at(const orc_handle* h, int ig, int is) { return h->g[ig].s[is]; }

/*
 * One trajectory of calcTransmit (src/RTMCphon.f90:1627-1836).
 * Surface indices are 0-based here (the reference's isurface-1); -1 plays the
 * role of the reference's isurface = 0 after a p-p event.
 * Returns EndSide: 1 (x-), 2 (x+) or 0 (lost).
 */
int trace_particle(const orc_handle* h, const Task& t, const Rng& rng, int64_t max_flights,
                   uint64_t* nflights, bool* capped, double* final_pos) {
  const double X = h->box[0], Y = h->box[1], Z = h->box[2];
  double d0, d1, e0, e1;
  /* createRandomPosition / createRandomDirectionPhi, :1845-1871 */
  rng.block(0, 0, &d0, &d1);
  double pos[3] = {0.0, d0 * Y * h->scope[0], d1 * Z * h->scope[1]};
  rng.block(0, 1, &e0, &e1);
  double sphi, cphi;
  orc::sincos_2pi(e0, &sphi, &cphi);
  double dir[3] = {t.cth, t.sth * cphi, t.sth * sphi};
  int EndSide = (dir[0] <= 0.0) ? 1 : 0;       /* StartSide = 1, :1635-1652 */
  int igrain = 0, isurface = 0, whichV = 0;     /* isurface = 1 (x-) in 1-based */
  if (h->ngrain > 0 && h->kind_grain == PTG_GRAIN_VORONOI) {
    /* findNearestIncidentGrain, :2100-2118 (0 when no grain is incident) */
    double dmin = 1.0e10;
    for (int ig = 1; ig <= h->ngrain; ++ig) {
      const Grain& g = h->g[ig];
      if (!g.incident) continue;
      double a = pos[0] - g.gen[0], b = pos[1] - g.gen[1], c = pos[2] - g.gen[2];
      double d2 = a * a + b * b + c * c;
      if (dmin > d2) { dmin = d2; whichV = ig; }
    }
  } else if (h->ngrain > 0 && h->kind_grain == PTG_GRAIN_BRICKS) {
    /* findIncidentCollisionGrain, :2131-2163: the last grain whose incident
       polygon contains the point wins, else the fill grain */
    bool found = false;
    for (int ig = 1; ig <= h->ngrain; ++ig) {
      const Grain& g = h->g[ig];
      if (!g.incident) continue;
      for (const Surf& s : g.s) {
        if (!s.incident) continue;
        if (inside_polygon(s, pos)) { whichV = ig; found = true; break; }
      }
    }
    if (!found) whichV = h->igrain_fill;
  }
  const bool ballistic = (t.lambda == BALLISTIC);
  double FreePath = ballistic ? BALLISTIC : -t.lambda * orc::log_pos(e1);
  uint64_t flight = 0;
  *capped = false;
  while (EndSide == 0) {
    /* isInsideBox (verbose >= 1), :1695-1703 */
    if (!(pos[0] >= 0.0 - SMALL_VAL && pos[0] <= X + SMALL_VAL && pos[1] >= 0.0 - SMALL_VAL &&
          pos[1] <= Y + SMALL_VAL && pos[2] >= 0.0 - SMALL_VAL && pos[2] <= Z + SMALL_VAL))
      break;
    if ((int64_t)flight >= max_flights) { *capped = true; break; }
    ++flight;
    const uint32_t fl = (uint32_t)flight;
    /* findCollisionSurface, :1989-2096 */
    double distance = 1.0e10;
    int ig_min = igrain, is_min = isurface;
    for (int pass = 0; pass < 2; ++pass) {
      int ig = (pass == 0) ? 0 : whichV;
      if (pass == 1 && whichV == 0) break;
      const Grain& g = h->g[ig];
      for (size_t is = 0; is < g.s.size(); ++is) {
        const Surf& s = g.s[is];
        if (!s.internal) continue;
        double L;
        if (surface_distance(h, pos, dir, s, &L) && distance > L) {
          distance = L; ig_min = ig; is_min = (int)is;
        }
      }
    }
    igrain = ig_min; isurface = is_min;
    int Jreflect = 1;
    bool pp = false;
    if (FreePath < distance) {
      /* intrinsic scattering, :1735-1742 and createRandomDirectionAllSphere :2192-2204 */
      distance = FreePath;
      for (int d = 0; d < 3; ++d) pos[d] = pos[d] + distance * dir[d];
      rng.block(fl, 0, &d0, &d1);
      double ct = d0 * 2.0 - 1.0;
      double sp, cp;
      orc::sincos_2pi(d1, &sp, &cp);
      double st = sqrt(1.0 - ct * ct);
      dir[0] = ct; dir[1] = st * cp; dir[2] = st * sp;
      igrain = 0; isurface = -1;
      pp = true;
    } else {
      for (int d = 0; d < 3; ++d) pos[d] = pos[d] + distance * dir[d];
      if (isurface < 0) {
        /* no surface found right after a p-p event: the reference would read
           vsurface(0) (out of bounds); the phonon is counted as lost */
        break;
      } else if (igrain == 0 && isurface == 0) {
        EndSide = 1;
      } else if (igrain == 0 && isurface == 1) {
        EndSide = 2;
      } else if (igrain == 0 && h->face_kind[isurface] == PTG_FACE_PERIODIC) {
        /* extension: periodic box face, wrap to the opposite face */
        int ax = isurface >> 1;
        double Lax = h->box[ax];
        if ((isurface & 1) == 0) pos[ax] = pos[ax] + Lax;
        else pos[ax] = pos[ax] - Lax;
      } else {
        const Surf& s = surf_at(h, igrain, isurface);
        rng.block(fl, 0, &d0, &d1);
        double od = 0.0;
        if (needs_omega_draw(h, s)) { double x; rng.block(fl, 2, &od, &x); }
        if (d0 <= s.spec) {
          /* reflectSpecular, :2275-2328 */
          double thr = transmit_threshold(h, s, t, od);
          if (d1 <= thr) {
            Jreflect = 0;
          } else {
            double N[3];
            surface_normal(s, pos, N);
            if (dot3(N, dir) < 0) for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
            double dn = dot3(N, dir);
            for (int d = 0; d < 3; ++d) dir[d] = dir[d] - 2.0 * N[d] * dn;
            Jreflect = 1;
          }
        } else {
          /* reflectDiffusive, :2332-2380 */
          double N[3], Rm[9];
          surface_normal(s, pos, N);
          if (dot3(N, dir) < 0.0) for (int d = 0; d < 3; ++d) N[d] = -1.0 * N[d];
          surface_rotation(s, pos, Rm);
          /* createRandomDirectionSemiSphere, :2208-2221 */
          double f0, f1;
          rng.block(fl, 1, &f0, &f1);
          double sint = sqrt(d1);
          double cost = sqrt(1.0 - sint * sint);
          double sp, cp;
          orc::sincos_2pi(f0, &sp, &cp);
          double td[3] = {sint * cp, sint * sp, cost};
          double v[3];
          for (int i = 0; i < 3; ++i) v[i] = Rm[i] * td[0] + Rm[3 + i] * td[1] + Rm[6 + i] * td[2];
          if (dot3(dir, N) > 0.0) {
            for (int i = 0; i < 3; ++i) dir[i] = -v[i];
          } else {
            for (int i = 0; i < 3; ++i) dir[i] = v[i];
          }
          if (dot3(dir, N) > 0.0) for (int i = 0; i < 3; ++i) dir[i] = -1.0 * dir[i];
          double thr = transmit_threshold(h, s, t, od);
          if (f1 <= thr) {
            for (int i = 0; i < 3; ++i) dir[i] = -dir[i];
            Jreflect = 0;
          } else {
            Jreflect = 1;
          }
        }
      }
    }
    /* move forward by a little, :1776-1780 */
    for (int d = 0; d < 3; ++d) pos[d] = pos[d] + 1.0e-7 * dir[d];
    /* free path update, :1783-1790 */
    if (ballistic) {
      FreePath = BALLISTIC;
    } else {
      FreePath = FreePath - distance;
      if (FreePath < 1.0e-10) {
        double r0, r1;
        if (pp) { rng.block(fl, 1, &r0, &r1); FreePath = -t.lambda * orc::log_pos(r0); }
        else { rng.block(fl, 2, &r0, &r1); FreePath = -t.lambda * orc::log_pos(r1); }
      }
    }
    if (Jreflect == 0) whichV = surf_at(h, igrain, isurface).grain_outside;
  }
  *nflights = flight;
  if (final_pos) for (int d = 0; d < 3; ++d) final_pos[d] = pos[d];
  return EndSide;
}

int64_t ntask_of(const orc_handle* h, const ptg_run* r) {
  int64_t nm = (int64_t)h->nb * h->nk;
  int64_t ns = (r->kind_mfp == PTG_MFP_GRID) ? r->nmfp : 1;
  return nm * ns * (r->nangle - 1);
}

bool run_valid(const orc_handle* h, const ptg_run* r) {
  if (!r || r->nangle < 3 || (r->nangle % 2) == 0 || r->np < 1 || r->nranks < 1 || r->rank < 0 ||
      r->rank >= r->nranks)
    return false;
  if (r->kind_mfp == PTG_MFP_GRID && (r->nmfp < 1 || !r->mfp_grid_nm)) return false;
  if (r->kind_mfp < 1 || r->kind_mfp > 3) return false;
  if (h->nb < 1 || h->nk < 1) return false;
  return true;
}

/* Task description from the ptg_run numbering. */
Task task_of(const orc_handle* h, const ptg_run* r, int64_t task) {
  int64_t nm = (int64_t)h->nb * h->nk;
  int64_t ns = (r->kind_mfp == PTG_MFP_GRID) ? r->nmfp : 1;
  int64_t m = task % nm;
  int64_t rest = task / nm;
  int64_t s = rest % ns;
  int64_t ia = rest / ns;
  Task t;
  t.ib = (int)(m % h->nb);
  t.ik = (int)(m / h->nb);
  t.omega = h->omega[m];
  double theta = 0.0 + (double)ia / (double)(r->nangle - 1) * M_PI_2_D;
  t.cth = cos(theta);
  t.sth = sin(theta);
  double scale = (r->scatter_scale > 0.0) ? r->scatter_scale : 1.0;
  if (r->kind_mfp == PTG_MFP_MATTHIESSEN) {
    t.lambda = BALLISTIC;
  } else if (r->kind_mfp == PTG_MFP_GRID) {
    t.lambda = r->mfp_grid_nm[s];
  } else {
    double tau_s = h->tau[m] * 1.0e-12 * (h->rtemp / r->temperature);
    t.lambda = tau_s * h->vel[m] * 1.0e9 / scale;
  }
  return t;
}

Rng rng_of(const ptg_run* r, uint64_t sample) {
  Rng g;
  g.k0 = (uint32_t)r->seed;
  g.k1 = (uint32_t)(r->seed >> 32);
  g.c1 = ((uint32_t)r->stream) << 8;
  g.slo = (uint32_t)sample;
  g.shi = (uint32_t)(sample >> 32);
  return g;
}

}  // namespace

extern "C" {

int64_t orc_ntask(const orc_handle* h, const ptg_run* run) {
  if (!h || !run) return -1;
  return ntask_of(h, run);
}

int orc_run_counts(orc_handle* h, const ptg_run* run, int64_t max_flights, int32_t ref_quirks,
                   int32_t nthreads, const int64_t* subset, int64_t nsubset, uint64_t* counts,
                   uint64_t* lost, orc_result* res) {
  if (!h || !run_valid(h, run)) return PTG_ERR_INVALID;
  if (max_flights <= 0) max_flights = 2147483647LL;
  int64_t ntask = ntask_of(h, run);
  int64_t nwork = subset ? nsubset : ntask;
  if (counts) memset(counts, 0, sizeof(uint64_t) * ntask);
  if (lost) memset(lost, 0, sizeof(uint64_t) * ntask);
  uint64_t tot_flights = 0, tot_lost = 0, tot_capped = 0, tot_samples = 0;
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(static) num_threads(nt) \
    reduction(+ : tot_flights, tot_lost, tot_capped, tot_samples)
  for (int64_t w = 0; w < nwork; ++w) {
    int64_t task = subset ? subset[w] : w;
    if (task < 0 || task >= ntask) continue;
    Task t = task_of(h, run, task);
    uint64_t c = 0, l = 0;
    if (t.lambda > 0.0) {
      for (int64_t p = run->rank; p < run->np; p += run->nranks) {
        uint64_t sample = (uint64_t)task * (uint64_t)run->np + (uint64_t)p;
        Rng rng = rng_of(run, sample);
        uint64_t nf = 0;
        bool capped = false;
        int es = trace_particle(h, t, rng, max_flights, &nf, &capped, nullptr);
        tot_flights += nf;
        tot_samples += 1;
        if (es == 2) c += 1;
        if (es == 0) {
          l += 1;
          if (capped) tot_capped += 1;
          if (ref_quirks) c += 1;  /* StartSide(1) /= EndSide(0), :1833 */
        }
      }
    }
    if (counts) counts[task] = c;
    if (lost) lost[task] = l;
    tot_lost += l;
  }
  auto t1 = std::chrono::steady_clock::now();
  if (res) {
    res->flights = tot_flights; res->lost = tot_lost; res->capped = tot_capped;
    res->samples = tot_samples;
    res->seconds = std::chrono::duration<double>(t1 - t0).count();
    res->threads = nt;
  }
  return PTG_OK;
}

int orc_replay_task(orc_handle* h, const ptg_run* run, int64_t task, int64_t max_flights,
                    int32_t* end_side, uint32_t* flights, double* final_pos) {
  if (!h || !run_valid(h, run)) return PTG_ERR_INVALID;
  if (task < 0 || task >= ntask_of(h, run)) return PTG_ERR_INVALID;
  if (max_flights <= 0) max_flights = 2147483647LL;
  Task t = task_of(h, run, task);
  int64_t j = 0;
  for (int64_t p = run->rank; p < run->np; p += run->nranks, ++j) {
    uint64_t sample = (uint64_t)task * (uint64_t)run->np + (uint64_t)p;
    Rng rng = rng_of(run, sample);
    uint64_t nf = 0;
    bool capped = false;
    double fp[3] = {0, 0, 0};
    int es = (t.lambda > 0.0) ? trace_particle(h, t, rng, max_flights, &nf, &capped, fp) : 0;
    if (end_side) end_side[j] = es;
    if (flights) flights[j] = (uint32_t)nf;
    if (final_pos) for (int d = 0; d < 3; ++d) final_pos[3 * j + d] = fp[d];
  }
  return PTG_OK;
}

/*
 * effectiveMFP (src/RTMCphon.f90:2418-2451) and the kappa sum of fileoutput
 * (:2645-2755), followed by the extensions: standard errors from the binomial
 * variance of each task and the flux-weighted per-bin transmission.
 */
int orc_kappa_from_counts(orc_handle* h, const ptg_run* run, const uint64_t* counts,
                          ptg_kappa_out* out) {
  if (!h || !run_valid(h, run) || !counts || !out) return PTG_ERR_INVALID;
  const int nb = h->nb, nk = h->nk, na = run->nangle;
  const int ns = (run->kind_mfp == PTG_MFP_GRID) ? run->nmfp : 1;
  const int64_t nm = (int64_t)nb * nk;
  const double T = run->temperature;
  std::vector<double> vangle(na);
  for (int ia = 0; ia < na; ++ia) vangle[ia] = 0.0 + (double)ia / (double)(na - 1) * M_PI_2_D;
  const double dS = (vangle[1] - vangle[0]) / 3.0 * 3.0 * 0.5 * h->box[0];
  /* Simpson weights c_a (1,4,2,4,...,4,1) times sin*cos */
  std::vector<double> wsc(na, 0.0), ca(na, 0.0);
  for (int ia = 1; ia < na - 1; ia += 2) { ca[ia - 1] += 1.0; ca[ia] += 4.0; ca[ia + 1] += 1.0; }
  for (int ia = 0; ia < na; ++ia) wsc[ia] = sin(vangle[ia]) * cos(vangle[ia]);
  /* SEMFP(ik,ib,s) and its variance */
  std::vector<double> semfp((size_t)nm * ns), svar((size_t)nm * ns);
  std::vector<double> WT(na);
  for (int s = 0; s < ns; ++s) {
    for (int ik = 0; ik < nk; ++ik) {
      for (int ib = 0; ib < nb; ++ib) {
        int64_t m = ib + (int64_t)nb * ik;
        double var = 0.0;
        for (int ia = 0; ia < na; ++ia) {
          double tr = 0.0;
          if (ia < na - 1) {
            int64_t task = m + nm * (s + (int64_t)ns * ia);
            tr = (double)counts[task] / (double)run->np;
            double vt = tr * (1.0 - tr) / (double)run->np;
            double c = ca[ia] * wsc[ia];
            var += c * c * vt;
            if (out->transmit) out->transmit[task] = tr;
          } else if (out->transmit) {
            out->transmit[m + nm * (s + (int64_t)ns * ia)] = 0.0;
          }
          WT[ia] = sin(vangle[ia]) * cos(vangle[ia]) * tr;
        }
        double I = 0.0;
        for (int ia = 1; ia < na - 1; ia += 2) I = I + (WT[ia - 1] + 4.0 * WT[ia] + WT[ia + 1]);
        semfp[(size_t)m * ns + s] = I * dS;
        svar[(size_t)m * ns + s] = var * dS * dS;
      }
    }
  }
  /* fileoutput, nmaterial == 1 branch, on copies of the mode arrays */
  std::vector<double> om(h->omega), wt(h->weight), ta(h->tau), ve(h->vel), mf(nm);
  std::vector<int64_t> perm(nm);
  for (int64_t m = 0; m < nm; ++m) perm[m] = m;
  const double scale = (run->scatter_scale > 0.0) ? run->scatter_scale : 1.0;
  for (int64_t m = 0; m < nm; ++m) {
    ta[m] = ta[m] * 1.0e-12 * (h->rtemp / T);
    mf[m] = ta[m] * ve[m] / scale;
  }
  double wsum = 0.0;
  for (int64_t m = 0; m < nm; ++m) wsum += wt[m];
  const int nqfbz = (int)(wsum / nb);
  /* exchange sort by omega within each branch, :2658-2691 */
  for (int ii = 0; ii < nb; ++ii) {
    for (int jj = 0; jj < nk - 1; ++jj) {
      for (int kk = jj + 1; kk < nk; ++kk) {
        int64_t a = ii + (int64_t)nb * jj, b = ii + (int64_t)nb * kk;
        if (om[a] > om[b]) {
          std::swap(om[a], om[b]); std::swap(wt[a], wt[b]); std::swap(ta[a], ta[b]);
          std::swap(ve[a], ve[b]); std::swap(mf[a], mf[b]); std::swap(perm[a], perm[b]);
        }
      }
    }
  }
  std::vector<double> tc(nm), emfp(nm), dem(nm * ns, 0.0), cap(nm);
  for (int64_t m = 0; m < nm; ++m) {
    double x = HBAR * om[m] / (KB * T);
    if (x <= 1.0e-10) cap[m] = KB;
    else { double q = (x / 2) / sinh(x / 2); cap[m] = KB * (q * q); }
  }
  for (int64_t m = 0; m < nm; ++m) {
    int64_t src = perm[m];   /* SEMFP travels with the sort */
    const double* S = &semfp[(size_t)src * ns];
    double E = 0.0;
    double* dE = &dem[(size_t)m * ns];
    if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
      if (mf[m] == 0.0) { E = S[0] * 1.0e-9; dE[0] = 1.0e-9; }
      else {
        E = 1.0 / (1.0 / mf[m] + 1.0 / (S[0] * 1.0e-9));
        double sm = S[0] * 1.0e-9;
        dE[0] = (sm > 0.0) ? 1.0e-9 * (E * E) / (sm * sm) : 1.0e-9;
      }
    } else if (run->kind_mfp == PTG_MFP_PER_MODE) {
      E = S[0] * 1.0e-9;
      dE[0] = 1.0e-9;
    } else {
      const double* g = run->mfp_grid_nm;
      if (mf[m] < g[0] * 1.0e-9) {
        E = S[0] * 1.0e-9 * mf[m] / (g[0] * 1.0e-9);
        dE[0] = 1.0e-9 * mf[m] / (g[0] * 1.0e-9);
      } else if (mf[m] > g[ns - 1] * 1.0e-9) {
        E = S[ns - 1] * 1.0e-9;
        dE[ns - 1] = 1.0e-9;
      } else {
        E = S[ns - 1] * 1.0e-9;   /* bulk MFP equal to the last grid point */
        dE[ns - 1] = 1.0e-9;
        for (int s = 0; s < ns - 1; ++s) {
          if (g[s] * 1.0e-9 <= mf[m] && mf[m] < g[s + 1] * 1.0e-9) {
            double ip = (mf[m] - g[s] * 1.0e-9) / ((g[s + 1] - g[s]) * 1.0e-9);
            E = S[s] * 1.0e-9 * (1.0 - ip) + S[s + 1] * 1.0e-9 * (ip);
            dE[ns - 1] = 0.0;
            dE[s] = 1.0e-9 * (1.0 - ip);
            dE[s + 1] = 1.0e-9 * ip;
            break;
          }
        }
      }
    }
    emfp[m] = E;
    tc[m] = cap[m] * wt[m] * E * ve[m] / 3 / h->vol / nqfbz;
  }
  double kappa = 0.0;
  for (int64_t m = 0; m < nm; ++m) kappa += tc[m];
  double kvar = 0.0;
  for (int64_t m = 0; m < nm; ++m) {
    double K = cap[m] * wt[m] * ve[m] / 3 / h->vol / nqfbz;
    int64_t src = perm[m];
    for (int s = 0; s < ns; ++s) {
      double g = K * dem[(size_t)m * ns + s];
      kvar += g * g * svar[(size_t)src * ns + s];
    }
  }
  out->kappa = kappa;
  out->kappa_stderr = sqrt(kvar);
  if (out->emfp_nm)
    for (int64_t m = 0; m < nm; ++m) out->emfp_nm[perm[m]] = emfp[m] * 1.0e9;
  if (run->nbins > 0 && (out->bin_T || out->bin_T_stderr)) {
    std::vector<double> sw(run->nbins, 0.0), swt(run->nbins, 0.0), sv(run->nbins, 0.0);
    const double lo = run->bin_omega_min, hi = run->bin_omega_max;
    for (int64_t m = 0; m < nm; ++m) {
      if (!(om[m] >= lo && om[m] <= hi) || !(hi > lo)) continue;
      int b = (int)floor((om[m] - lo) / (hi - lo) * run->nbins);
      if (b >= run->nbins) b = run->nbins - 1;
      if (b < 0) b = 0;
      double W = cap[m] * wt[m] * ve[m];
      int64_t src = perm[m];
      double tm, vm = 0.0;
      if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
        tm = semfp[(size_t)src * ns] / (0.75 * h->box[0]);
        vm = svar[(size_t)src * ns] / ((0.75 * h->box[0]) * (0.75 * h->box[0]));
      } else {
        tm = emfp[m] * 1.0e9 / (0.75 * h->box[0]);
        for (int s = 0; s < ns; ++s) {
          double g = dem[(size_t)m * ns + s] * 1.0e9 / (0.75 * h->box[0]);
          vm += g * g * svar[(size_t)src * ns + s];
        }
      }
      sw[b] += W; swt[b] += W * tm; sv[b] += W * W * vm;
    }
    for (int b = 0; b < run->nbins; ++b) {
      if (out->bin_T) out->bin_T[b] = sw[b] > 0 ? swt[b] / sw[b] : 0.0;
      if (out->bin_T_stderr) out->bin_T_stderr[b] = sw[b] > 0 ? sqrt(sv[b]) / sw[b] : 0.0;
    }
  }
  return PTG_OK;
}

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t o[4]) {
  orc::Philox4 p = orc::philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  for (int i = 0; i < 4; ++i) o[i] = p.v[i];
}
double orc_log(double x) { return orc::log_pos(x); }
void orc_sincos2pi(double u, double* s, double* c) { orc::sincos_2pi(u, s, c); }

}  // extern "C"

/* ------------------------------------------------------------------------ */
/* fileoutput's files, src/RTMCphon.f90:2601-2881, restated with the
   reference's exchange sorts and gfortran's rendering of its edit
   descriptors (Iw right-justified or asterisks; Fw.d; Ew.d as 0.ddE+xx,
   +xxx past two exponent digits). */
namespace {

std::string orc_rjust(const std::string& s, int w) {
  return (w > 0 && (int)s.size() < w) ? std::string(w - s.size(), ' ') + s : s;
}

std::string orc_I(long long v, int w) {
  char b[64];
  snprintf(b, sizeof(b), "%lld", v);
  std::string s = b;
  return (int)s.size() > w ? std::string(w, '*') : orc_rjust(s, w);
}

std::string orc_F(double v, int w, int d) {
  char b[512];
  snprintf(b, sizeof(b), "%.*f", d, v);
  std::string s = b;
  if (w == 0) return s;
  if ((int)s.size() > w && s.compare(0, 2, "0.") == 0) s.erase(0, 1);
  if ((int)s.size() > w && s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
  return (int)s.size() > w ? std::string(w, '*') : orc_rjust(s, w);
}

std::string orc_E(double v, int w, int d) {
  /* d significant digits of |v| as 0.d1..dd * 10^e */
  std::string digits(d, '0');
  int e = 0;
  if (v != 0.0) {
    char b[128];
    snprintf(b, sizeof(b), "%.*e", d - 1, fabs(v));
    std::string t = b;
    size_t ep = t.find('e');
    std::string m = t.substr(0, ep);
    m.erase(std::remove(m.begin(), m.end(), '.'), m.end());
    digits = m;
    e = atoi(t.c_str() + ep + 1) + 1;
  }
  char x[16];
  if (e >= -99 && e <= 99) snprintf(x, sizeof(x), "E%+03d", e);
  else snprintf(x, sizeof(x), "%+04d", e);
  const std::string sg = (v < 0.0) ? "-" : "";
  std::string s = sg + "0." + digits + x;
  if ((int)s.size() > w) s = sg + "." + digits + x;
  return (int)s.size() > w ? std::string(w, '*') : orc_rjust(s, w);
}

}  // namespace

extern "C" int orc_write_outputs(orc_handle* h, const char* geofile, const ptg_run* run,
                                 const uint64_t* counts) {
  if (!h || !geofile || !run_valid(h, run) || !counts) return PTG_ERR_INVALID;
  const int nb = h->nb, nk = h->nk, na = run->nangle;
  const int nmfp = (run->kind_mfp == PTG_MFP_GRID) ? run->nmfp : 1;
  const int64_t nm = (int64_t)nb * nk;
  const double T = run->temperature;
  /* effectiveMFP: SEMFP(ik, ib, s) */
  std::vector<double> vangle(na), WT(na);
  for (int ia = 0; ia < na; ++ia) vangle[ia] = 0.0 + (double)ia / (double)(na - 1) * M_PI_2_D;
  const double dS = (vangle[1] - vangle[0]) / 3.0 * 3.0 * 0.5 * h->box[0];
  std::vector<double> SEMFP((size_t)nk * nb * nmfp);
  auto sidx = [&](int ik, int ib, int s) { return (size_t)ik + (size_t)nk * ((size_t)ib + (size_t)nb * s); };
  for (int s = 0; s < nmfp; ++s)
    for (int ik = 0; ik < nk; ++ik)
      for (int ib = 0; ib < nb; ++ib) {
        for (int ia = 0; ia < na; ++ia) {
          const double tr = (ia < na - 1)
              ? (double)counts[ib + (int64_t)nb * ik + nm * (s + (int64_t)nmfp * ia)] / (double)run->np
              : 0.0;
          WT[ia] = sin(vangle[ia]) * cos(vangle[ia]) * tr;
        }
        double I = 0.0;
        for (int ia = 2; ia <= na - 1; ia += 2) I = I + (WT[ia - 2] + 4.0 * WT[ia - 1] + WT[ia]);
        SEMFP[sidx(ik, ib, s)] = I * dS;
      }
  std::string g = geofile;
  size_t c = g.rfind('/');
  if (c == std::string::npos) c = g.rfind('\\');
  const std::string pre = (c == std::string::npos) ? "" : g.substr(0, c + 1);
  std::string f41 = "# Datatype = thermalproperty\n";
  f41 += "# Incident_Phonon                               =   " + orc_I(run->np, 6) + "\n";
  if (h->nmaterial > 1) {
    f41 += "# Effective_MeanFreePath [nm]       = " + orc_E(SEMFP[0], 20, 10) + "\n";
    FILE* f = fopen((pre + "thermalproperty.out").c_str(), "w");
    if (!f) return PTG_ERR_IO;
    fputs(f41.c_str(), f);
    fclose(f);
    return PTG_OK;
  }
  double ssum = 0.0;
  for (double v : SEMFP) ssum += v;
  f41 += "# Averaged Effective_MeanFreePath [nm]          = " +
         orc_F(ssum / (nb * nk * nmfp), 20, 10) + "\n";
  /* anphon copies (ii = branch, jj = k-point), tau rescale, MFP */
  const double scale = (run->scatter_scale > 0.0) ? run->scatter_scale : 1.0;
  std::vector<double> om(h->omega), wt(h->weight), ta(h->tau), ve(h->vel), mf(nm);
  auto A = [&](int ii, int jj) { return (size_t)ii + (size_t)nb * jj; };
  for (int jj = 0; jj < nk; ++jj)
    for (int ii = 0; ii < nb; ++ii) {
      ta[A(ii, jj)] = ta[A(ii, jj)] * 1.0e-12 * (h->rtemp / T);
      mf[A(ii, jj)] = ta[A(ii, jj)] * ve[A(ii, jj)] / scale;
    }
  double wsum = 0.0;
  for (double v : wt) wsum += v;
  const int nqfbz = (int)(wsum / nb);
  for (int ii = 0; ii < nb; ++ii)
    for (int jj = 0; jj < nk - 1; ++jj)
      for (int kk = jj + 1; kk < nk; ++kk)
        if (om[A(ii, jj)] > om[A(ii, kk)]) {
          std::swap(om[A(ii, jj)], om[A(ii, kk)]);
          std::swap(wt[A(ii, jj)], wt[A(ii, kk)]);
          std::swap(ta[A(ii, jj)], ta[A(ii, kk)]);
          std::swap(ve[A(ii, jj)], ve[A(ii, kk)]);
          std::swap(mf[A(ii, jj)], mf[A(ii, kk)]);
          for (int s = 0; s < nmfp; ++s) std::swap(SEMFP[sidx(jj, ii, s)], SEMFP[sidx(kk, ii, s)]);
        }
  std::vector<double> cap(nm), EMFP(nm), TC(nm);
  for (int ii = 0; ii < nb; ++ii)
    for (int jj = 0; jj < nk; ++jj) {
      const double x = HBAR * om[A(ii, jj)] / (KB * T);
      cap[A(ii, jj)] = (x <= 1.0e-10) ? KB : KB * (((x / 2) / sinh(x / 2)) * ((x / 2) / sinh(x / 2)));
    }
  for (int ii = 0; ii < nb; ++ii)
    for (int jj = 0; jj < nk; ++jj) {
      const double m = mf[A(ii, jj)];
      double E;
      if (run->kind_mfp == PTG_MFP_MATTHIESSEN) {
        E = (m == 0.0) ? SEMFP[sidx(jj, ii, 0)] * 1.0e-9
                       : 1.0 / (1.0 / m + 1.0 / (SEMFP[sidx(jj, ii, 0)] * 1.0e-9));
      } else if (run->kind_mfp == PTG_MFP_PER_MODE) {
        E = SEMFP[sidx(jj, ii, 0)] * 1.0e-9;
      } else {
        const double* v = run->mfp_grid_nm;
        E = SEMFP[sidx(jj, ii, nmfp - 1)] * 1.0e-9;
        if (m < v[0] * 1.0e-9) {
          E = SEMFP[sidx(jj, ii, 0)] * 1.0e-9 * m / (v[0] * 1.0e-9);
        } else if (!(m > v[nmfp - 1] * 1.0e-9)) {
          for (int s = 0; s < nmfp - 1; ++s)
            if (v[s] * 1.0e-9 <= m && m < v[s + 1] * 1.0e-9) {
              const double ip = (m - v[s] * 1.0e-9) / ((v[s + 1] - v[s]) * 1.0e-9);
              E = SEMFP[sidx(jj, ii, s)] * 1.0e-9 * (1.0 - ip) + SEMFP[sidx(jj, ii, s + 1)] * 1.0e-9 * ip;
              break;
            }
        }
      }
      EMFP[A(ii, jj)] = E;
      TC[A(ii, jj)] = cap[A(ii, jj)] * wt[A(ii, jj)] * EMFP[A(ii, jj)] * ve[A(ii, jj)] / 3 / h->vol / nqfbz;
    }
  double ktot = 0.0;
  for (size_t i = 0; i < (size_t)nm; ++i) ktot += TC[i];  /* column-major sum(TC(:,:)) */
  f41 += "# Thermal_conductivity@" + orc_F(T, 0, 6) + "K [W m-1 K-1]  = " + orc_F(ktot, 20, 10) + "\n";
  {
    FILE* f = fopen((pre + "thermalproperty.out").c_str(), "w");
    if (!f) return PTG_ERR_IO;
    fputs(f41.c_str(), f);
    fclose(f);
  }
  /* effectiveMFP.out */
  struct Rec { int ib, ik; double bulk, eff, cond, acc; };
  std::vector<Rec> vd;
  for (int ii = 0; ii < nb; ++ii)
    for (int jj = 0; jj < nk; ++jj)
      vd.push_back({ii + 1, jj + 1, mf[A(ii, jj)], EMFP[A(ii, jj)], TC[A(ii, jj)], 0.0});
  const int cf = (int)vd.size();
  for (int ii = 0; ii < cf; ++ii)
    for (int jj = ii + 1; jj < cf; ++jj)
      if (vd[ii].eff > vd[jj].eff) std::swap(vd[ii], vd[jj]);
  vd[0].acc = vd[0].cond;
  for (int ii = 1; ii < cf; ++ii) vd[ii].acc = vd[ii].cond + vd[ii - 1].acc;
  {
    FILE* f = fopen((pre + "effectiveMFP.out").c_str(), "w");
    if (!f) return PTG_ERR_IO;
    fputs("# Datatype = Effective Mean Free Path of phonon.\n", f);
    fputs("# data are sorted by effective MFP in ascending order.\n", f);
    fprintf(f, "#   total branches: %s\n", orc_I(nb, 3).c_str());
    fprintf(f, "#   total Kpoints:  %s\n", orc_I(nk, 3).c_str());
    fputs("#\n", f);
    fputs("# branch, kpoint, bulk MFP[nm], effective MFP[nm], ThermalConductivity, and its accumulated[W m-1 K-1].\n", f);
    for (const Rec& r : vd)
      fprintf(f, "%s%s%s%s%s%s\n", orc_I(r.ib, 5).c_str(), orc_I(r.ik, 5).c_str(),
              orc_E(r.bulk * 1.0e9, 15, 6).c_str(), orc_E(r.eff * 1.0e9, 15, 6).c_str(),
              orc_E(r.cond, 15, 6).c_str(), orc_E(r.acc, 15, 6).c_str());
    fclose(f);
  }
  /* phononconductivity.out */
  std::vector<double> so;
  for (int ii = 0; ii < nb; ++ii)
    for (int jj = 0; jj < nk; ++jj) {
      bool dup = false;
      for (double v : so) if (v == om[A(ii, jj)]) { dup = true; break; }
      if (!dup) so.push_back(om[A(ii, jj)]);
    }
  const int nf = (int)so.size();
  for (int ii = 0; ii < nf - 1; ++ii)
    for (int jj = ii + 1; jj < nf; ++jj)
      if (so[ii] > so[jj]) std::swap(so[ii], so[jj]);
  FILE* f = fopen((pre + "phononconductivity.out").c_str(), "w");
  if (!f) return PTG_ERR_IO;
  fputs("# Datatype = phononconductivity\n", f);
  fprintf(f, "# Nb = %s\n", orc_I(nf - 1, 6).c_str());
  fprintf(f, "# Nbranch = %s\n", orc_I(nb, 4).c_str());
  fputs("# omega, fluxphononout(1:Nbranch)\n", f);
  for (int ii = 0; ii < nf - 1; ++ii) {
    fputs(orc_E(so[ii], 20, 10).c_str(), f);
    for (int jj = 0; jj < nb; ++jj) {
      double k = 0.0;
      for (int kk = 0; kk < nk; ++kk)
        if (om[A(jj, kk)] == so[ii]) k = k + TC[A(jj, kk)];
      fputs(orc_E(k, 20, 10).c_str(), f);
    }
    fputs("\n", f);
  }
  fclose(f);
  return PTG_OK;
}

/* GammaDeterm with ModeNum = 1, src/RTMCphon.f90:2499-2560, on the handle's
   spectrum (the material's anphon). */
extern "C" int orc_gamma_from_tbc(orc_handle* h, double temperature, double TBC, double* gamma) {
  if (!h || !gamma) return PTG_ERR_INVALID;
  const int nbranch = h->nb, nkpoint = h->nk;
  std::vector<double> cap((size_t)nbranch * nkpoint, 0.0);
  double wsum = 0.0;
  for (double w : h->weight) wsum += w;
  const int nqfbz = (int)(wsum / nbranch);
  auto X = [&](const std::vector<double>& a, int b, int k) { return a[(size_t)b + (size_t)nbranch * k]; };
  for (int ii = 0; ii < nkpoint; ++ii)
    for (int jj = 0; jj < nbranch; ++jj) {
      const double tmpX = HBAR * X(h->omega, jj, ii) / (KB * temperature);
      cap[(size_t)jj + (size_t)nbranch * ii] =
          (tmpX <= 1.0e-10) ? KB : KB * (((tmpX / 2) / sinh(tmpX / 2)) * ((tmpX / 2) / sinh(tmpX / 2)));
    }
  const double maxOmega = h->max_omega;
  double tmpGamma = 1.0e-2;
  for (int it = 1; it <= 10000; ++it) {
    double tmpTBC = 0.0, tmpTBCa = 0.0, tmpdTBC = 0.0;
    for (int jj = 0; jj < nkpoint; ++jj)
      for (int kk = 0; kk < nbranch; ++kk) {
        const double tmpH = 1 / (tmpGamma * (X(h->omega, kk, jj) / maxOmega) + 1);
        tmpTBC = tmpTBC + X(h->weight, kk, jj) * X(cap, kk, jj) * X(h->vel, kk, jj) * tmpH / 2 / h->vol / nqfbz;
      }
    for (int jj = 0; jj < nkpoint; ++jj)
      for (int kk = 0; kk < nbranch; ++kk) {
        const double tmpH = 1;
        tmpTBCa = tmpTBCa + X(h->weight, kk, jj) * X(cap, kk, jj) * X(h->vel, kk, jj) * tmpH / 2 / h->vol / nqfbz;
      }
    for (int jj = 0; jj < nkpoint; ++jj)
      for (int kk = 0; kk < nbranch; ++kk) {
        const double den = tmpGamma * (X(h->omega, kk, jj) / maxOmega) + 1;
        const double tmpH = -(X(h->omega, kk, jj) / maxOmega) / (den * den);
        tmpdTBC = tmpdTBC + X(h->weight, kk, jj) * X(cap, kk, jj) * X(h->vel, kk, jj) * tmpH / 2 / h->vol / nqfbz;
      }
    const double tmpF = tmpTBC / (1 - tmpTBC / tmpTBCa) - TBC;
    const double one = 1 - tmpTBC / tmpTBCa;
    const double tmpdF = tmpdTBC / (one * one);
    const double differential = tmpF / tmpdF;
    if (fabs(differential) <= 1.0e-6) break;
    tmpGamma = tmpGamma - differential;
  }
  *gamma = tmpGamma;
  return tmpGamma < 0.0 ? PTG_ERR_INVALID : PTG_OK;
}
