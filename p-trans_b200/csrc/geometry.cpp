/*
 * geometry.cpp - host construction of the built geometry from the raw
 * structure description, plus validation of caller-built geometry.
 *
 * Restates src/RTMCphon.f90:
 *   setupBoxGrain              :1253-1332  (box grain 0, six outward quads)
 *   loadGeometry grain loop    :968-1171   (facets, incident / internal flags,
 *                                           material_to, grain_to, specularity)
 *   setupFillGrain             :1336-1398  (bricks: reversed copies)
 *   setupSurfaceTransmissivity :1402-1429  (stored as kind + scalar)
 *   setupSurfaceGeometry       :1433-1491  (centre, averaged normal, frame)
 */
#include <math.h>
#include <algorithm>
#include <string.h>

#include <string>
#include <vector>

#include "ptg_internal.h"

namespace ptg {

namespace {

struct Surf {
  int32_t shape = PTG_SHAPE_POLYGON, nvertex = 0;
  std::vector<double> v;  /* closed: nvertex+1 points */
  double normal[3] = {0, 0, 0}, tangent[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double center[3] = {0, 0, 0}, radius = 0;
  int32_t kind_trans = PTG_TRANS_VALUE, mat1 = 0, mat2 = 0;
  double spec = 0, tparam = 0;
  int32_t gin = 0, gout = 0, internal = 1, incident = 0;
};

struct GrainRec {
  int32_t incident = 0;
  double gen[3] = {0, 0, 0};
  std::vector<Surf> s;
};

inline double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Frame whose third column is n: (1,0,0),(0,1,0) when n is along z, else
   t2 = (-ny, nx, 0)/|.|, t1 = t2 x n (src/RTMCphon.f90:1471-1487). */
void frame_from_normal(const double* n, double* t) {
  t[6] = n[0]; t[7] = n[1]; t[8] = n[2];
  if (fabs(n[2]) == 1.0 || (n[0] * n[0] == 0.0 && n[1] * n[1] == 0.0)) {
    t[0] = 1; t[1] = 0; t[2] = 0;
    t[3] = 0; t[4] = 1; t[5] = 0;
    return;
  }
  double q = sqrt(n[0] * n[0] + n[1] * n[1]);
  t[3] = -n[1] / q;
  t[4] = n[0] / q;
  t[5] = 0.0;
  cross(&t[3], &t[6], &t[0]);
}

/* Centre = vertex mean; normal = mean of the unit normals of the nvertex
   consecutive vertex triples (src/RTMCphon.f90:1440-1465). */
void polygon_setup(Surf& s) {
  const int n = s.nvertex;
  const double* v = s.v.data();
  double c[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] = c[d] + v[3 * i + d];
  for (int d = 0; d < 3; ++d) s.center[d] = 1.0 / n * c[d];
  double acc[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    /* triple (i, i+1, i+2) on the closed list; the last one is (n-1, n, 1) */
    const double* p0 = v + 3 * (i < n - 1 ? i : n - 1);
    const double* p1 = v + 3 * (i < n - 1 ? i + 1 : n);
    const double* p2 = v + 3 * (i < n - 1 ? i + 2 : 1);
    double a[3], b[3], x[3];
    for (int d = 0; d < 3; ++d) { a[d] = p1[d] - p0[d]; b[d] = p2[d] - p0[d]; }
    cross(a, b, x);
    double len = sqrt(dot(x, x));
    for (int d = 0; d < 3; ++d) acc[d] = acc[d] + x[d] / len;
  }
  for (int d = 0; d < 3; ++d) s.normal[d] = 1.0 / n * acc[d];
  frame_from_normal(s.normal, s.tangent);
}

/* Twelve-uniform Gaussian of normal_distribution (src/RTMCphon.f90:1188-1199)
   drawn from Philox4x32-10: key = seed, counter = (j, 0x464C, surface, 0). */
uint32_t mulhi(uint32_t a, uint32_t b, uint32_t* lo) {
  uint64_t p = (uint64_t)a * b;
  *lo = (uint32_t)p;
  return (uint32_t)(p >> 32);
}
void philox_host(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint32_t lo0, lo1;
    uint32_t hi0 = mulhi(0xD2511F53u, c[0], &lo0);
    uint32_t hi1 = mulhi(0xCD9E8D57u, c[2], &lo1);
    uint32_t a = hi1 ^ c[1] ^ k0, b = hi0 ^ c[3] ^ k1;
    c[0] = a; c[1] = lo1; c[2] = b; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}
double gaussian12(uint64_t seed, int32_t surf, double mean, double dev) {
  double sum = 0.0;
  for (uint32_t j = 0; j < 3; ++j) {
    uint32_t c[4] = {j, 0x464Cu, (uint32_t)surf, 0u};
    philox_host(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int w = 0; w < 4; ++w) sum = sum + ((double)c[w] + 0.5) * (1.0 / 4294967296.0);
  }
  return (sum - 6.0) * dev + mean;
}

bool table_ok(const ptg_model* m, int i2, int i1) {
  return i2 >= 1 && i2 <= m->nt2 + 1 && i1 >= 1 && i1 <= m->nt1 && m->tt_kind && m->tt_trans &&
         m->tt_spec;
}
size_t table_at(const ptg_model* m, int i2, int i1) {
  return (size_t)(i2 - 1) + (size_t)(m->nt2 + 1) * (size_t)(i1 - 1);
}

/* Interface properties of an internal surface from the material table. */
void interface_props(const ptg_model* m, Surf& s) {
  size_t k = table_at(m, s.mat2, s.mat1);
  s.spec = m->tt_spec[k];
  s.kind_trans = m->tt_kind[k];
  s.tparam = m->tt_trans[k];
}

bool finite3(const double* p) { return isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]); }

}  // namespace

void GeomSoA::make_view() {
  ptg_geometry& g = view;
  memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) g.box[d] = box[d];
  g.scope[0] = scope[0];
  g.scope[1] = scope[1];
  for (int f = 0; f < 6; ++f) g.face_kind[f] = face_kind[f];
  g.kind_grain = kind_grain;
  g.ngrain = ngrain;
  g.igrain_fill = igrain_fill;
  g.nmaterial = nmaterial;
  g.ngrain_total = ngrain_total();
  g.nsurf = nsurf();
  g.nvertex_total = (int32_t)(vertex.size() / 3);
  g.grain_begin = grain_begin.data();
  g.grain_incident = grain_incident.data();
  g.grain_generatrix = grain_generatrix.data();
  g.shape = shape.data();
  g.nvertex = nvertex.data();
  g.vertex_begin = vertex_begin.data();
  g.vertex = vertex.data();
  g.normal = normal.data();
  g.tangent = tangent.data();
  g.center = center.data();
  g.radius = radius.data();
  g.kind_trans = kind_trans.data();
  g.specularity = specularity.data();
  g.trans_param = trans_param.data();
  g.grain_inside = grain_inside.data();
  g.grain_outside = grain_outside.data();
  g.internal = internal.data();
  g.incident = incident.data();
  g.material1 = material1.data();
  g.material2 = material2.data();
}

static void flatten(const std::vector<GrainRec>& grains, GeomSoA* out) {
  out->grain_begin.clear();
  out->grain_incident.clear();
  out->grain_generatrix.clear();
  int32_t k = 0, vtx = 0;
  for (const GrainRec& g : grains) {
    out->grain_begin.push_back(k);
    out->grain_incident.push_back(g.incident);
    for (int d = 0; d < 3; ++d) out->grain_generatrix.push_back(g.gen[d]);
    for (const Surf& s : g.s) {
      out->shape.push_back(s.shape);
      out->nvertex.push_back(s.nvertex);
      out->vertex_begin.push_back(vtx);
      if (s.nvertex > 0) {
        out->vertex.insert(out->vertex.end(), s.v.begin(), s.v.end());
        vtx += s.nvertex + 1;
      }
      for (int d = 0; d < 3; ++d) out->normal.push_back(s.normal[d]);
      for (int d = 0; d < 9; ++d) out->tangent.push_back(s.tangent[d]);
      for (int d = 0; d < 3; ++d) out->center.push_back(s.center[d]);
      out->radius.push_back(s.radius);
      out->kind_trans.push_back(s.kind_trans);
      out->specularity.push_back(s.spec);
      out->trans_param.push_back(s.tparam);
      out->grain_inside.push_back(s.gin);
      out->grain_outside.push_back(s.gout);
      out->internal.push_back(s.internal);
      out->incident.push_back(s.incident);
      out->material1.push_back(s.mat1);
      out->material2.push_back(s.mat2);
      ++k;
    }
  }
  out->grain_begin.push_back(k);
  out->make_view();
}

int build_geometry(const ptg_model* m, GeomSoA* out, std::string* why) {
  if (!m || !out) { *why = "null model"; return PTG_ERR_INVALID; }
  if (m->ngrain < 1) {
    /* the reference scans "do ig=0,whichV,whichV", which needs a grain */
    *why = "ngrain must be >= 1";
    return PTG_ERR_INVALID;
  }
  if (m->kind_grain != PTG_GRAIN_VORONOI && m->kind_grain != PTG_GRAIN_BRICKS) {
    *why = "kind_grain must be voronoi (1) or bricks (2)";
    return PTG_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d)
    if (!(m->box[d] > 0.0) || !isfinite(m->box[d])) { *why = "box lengths must be > 0"; return PTG_ERR_INVALID; }
  if (m->nmaterial < 1) { *why = "nmaterial must be >= 1"; return PTG_ERR_INVALID; }
  if (m->face_kind[0] != PTG_FACE_REFERENCE || m->face_kind[1] != PTG_FACE_REFERENCE) {
    *why = "x faces are the heat baths and cannot be periodic";
    return PTG_ERR_INVALID;
  }
  for (int f = 2; f < 6; f += 2) {
    if (m->face_kind[f] != m->face_kind[f + 1]) {
      *why = "periodic faces come in pairs";
      return PTG_ERR_INVALID;
    }
  }
  const double X = m->box[0], Y = m->box[1], Z = m->box[2];
  const bool bricks = (m->kind_grain == PTG_GRAIN_BRICKS);
  const int32_t fill = bricks ? m->ngrain + 1 : -1;
  std::vector<GrainRec> grains(m->ngrain + 1 + (bricks ? 1 : 0));

  /* grain 0: the box, faces x-, x+, y-, y+, z-, z+ with outward normals */
  const double V[6][4][3] = {{{0, 0, 0}, {0, 0, Z}, {0, Y, Z}, {0, Y, 0}},
                             {{X, 0, 0}, {X, Y, 0}, {X, Y, Z}, {X, 0, Z}},
                             {{0, 0, 0}, {X, 0, 0}, {X, 0, Z}, {0, 0, Z}},
                             {{X, Y, 0}, {0, Y, 0}, {0, Y, Z}, {X, Y, Z}},
                             {{0, 0, 0}, {0, Y, 0}, {X, Y, 0}, {X, 0, 0}},
                             {{0, Y, Z}, {0, 0, Z}, {X, 0, Z}, {X, Y, Z}}};
  grains[0].s.resize(6);
  for (int f = 0; f < 6; ++f) {
    Surf& s = grains[0].s[f];
    s.nvertex = 4;
    s.v.resize(15);
    for (int i = 0; i < 5; ++i)
      for (int d = 0; d < 3; ++d) s.v[3 * i + d] = V[f][i & 3][d];
    polygon_setup(s);
    s.spec = m->cellspec[f];
    s.kind_trans = PTG_TRANS_VALUE;
    s.tparam = 0.0;
    s.gin = 0;
    s.gout = 0;
  }

  int fpos = 0, vpos = 0, mpos = 0;
  int32_t built = 6;
  for (int ig = 1; ig <= m->ngrain; ++ig) {
    ptg::alloc_check();  /* allocation-failure injection point (tests) */
    GrainRec& g = grains[ig];
    for (int d = 0; d < 3; ++d) g.gen[d] = m->grain_generatrix[3 * (ig - 1) + d];
    const int shape = bricks ? m->grain_shape[ig - 1] : PTG_SHAPE_POLYGON;
    if (shape < PTG_SHAPE_POLYGON || shape > PTG_SHAPE_CAPPED) {
      *why = "unknown grain shape";
      return PTG_ERR_INVALID;
    }
    if (shape == PTG_SHAPE_CAPPED && !m->grain_axis) {
      *why = "capped cylinders need grain_axis";
      return PTG_ERR_INVALID;
    }
    const int32_t mat1 = m->grain_material[ig - 1];
    if (mat1 < 1 || mat1 > m->nmaterial) { *why = "grain material out of range"; return PTG_ERR_INVALID; }
    const double radius = (shape == PTG_SHAPE_POLYGON) ? 0.0 : m->grain_diameter[ig - 1] * 0.5;
    if (shape != PTG_SHAPE_POLYGON && !(radius > 0.0)) { *why = "sphere/cylinder diameter must be > 0"; return PTG_ERR_INVALID; }
    const int nsurf = (shape == PTG_SHAPE_POLYGON) ? m->grain_nfacet[ig - 1] : 1;
    if (nsurf < 1) { *why = "a polygon grain needs facets"; return PTG_ERR_INVALID; }
    g.s.resize(nsurf);
    for (int is = 0; is < nsurf; ++is, ++mpos, ++built) {
      Surf& s = g.s[is];
      s.shape = shape;
      s.gin = ig;
      s.mat1 = mat1;
      for (int d = 0; d < 3; ++d) s.center[d] = g.gen[d];
      s.radius = radius;
      if (shape == PTG_SHAPE_POLYGON) {
        const int nv = m->facet_nvertex[fpos++];
        if (nv < 3) { *why = "a facet needs >= 3 vertices"; return PTG_ERR_INVALID; }
        s.nvertex = nv;
        s.v.resize(3 * (nv + 1));
        for (int i = 0; i < nv; ++i)
          for (int d = 0; d < 3; ++d) s.v[3 * i + d] = m->facet_vertex[3 * (vpos + i) + d];
        for (int d = 0; d < 3; ++d) s.v[3 * nv + d] = s.v[d];
        for (int i = 0; i < nv; ++i)
          if (!finite3(&s.v[3 * i])) { *why = "non-finite vertex"; return PTG_ERR_INVALID; }
        vpos += nv;
        polygon_setup(s);
        if (!finite3(s.normal)) { *why = "degenerate facet (zero area)"; return PTG_ERR_INVALID; }
        /* incident: every vertex at x <= 0; not internal: every vertex on
           or beyond one box face (src/RTMCphon.f90:1202-1246) */
        bool lo[3] = {true, true, true}, hi[3] = {true, true, true};
        for (int i = 0; i <= nv; ++i) {
          for (int d = 0; d < 3; ++d) {
            if (!(s.v[3 * i + d] <= 0.0)) lo[d] = false;
            if (!(s.v[3 * i + d] >= m->box[d])) hi[d] = false;
          }
        }
        if (lo[0]) { g.incident = 1; s.incident = 1; s.internal = 0; }
        if (lo[0] || hi[0] || lo[1] || hi[1] || lo[2] || hi[2]) s.internal = 0;
      } else {
        if (!finite3(s.center)) { *why = "non-finite centre"; return PTG_ERR_INVALID; }
        if (shape == PTG_SHAPE_CAPPED) {
          /* axis end points A = c - axis/2, B = c + axis/2, closed list */
          const double* ax = m->grain_axis + 3 * (ig - 1);
          if (!finite3(ax) || !(dot(ax, ax) > 0.0)) { *why = "capped cylinder axis must be > 0"; return PTG_ERR_INVALID; }
          s.nvertex = 2;
          s.v.resize(9);
          for (int d = 0; d < 3; ++d) {
            s.v[d] = s.center[d] - 0.5 * ax[d];
            s.v[3 + d] = s.center[d] + 0.5 * ax[d];
            s.v[6 + d] = s.v[d];
          }
        }
      }
      const int32_t mto = m->surf_material_to[mpos];
      s.gout = m->surf_grain_to[mpos];
      if (!s.internal) continue;
      if (mto == PTG_MATERIAL_INTERNAL) {
        s.mat2 = 1;
        s.gout = fill;
      } else {
        if (mto < 1 || mto > m->nmaterial) { *why = "material_to not a known material"; return PTG_ERR_INVALID; }
        s.mat2 = mto;
      }
      if (!table_ok(m, s.mat2, s.mat1)) { *why = "transmission table index out of range"; return PTG_ERR_INVALID; }
      interface_props(m, s);
      if (m->specfluc > 0.0) {
        s.spec = gaussian12(m->fluct_seed, built, s.spec, m->specfluc);
        if (s.spec < 0.0) s.spec = 0.0;
        if (s.spec > 1.0) s.spec = 1.0;
      }
      if (m->surf_spec) s.spec = m->surf_spec[mpos];
      if (s.gout < 0 || s.gout >= (int32_t)grains.size()) {
        *why = "grain_to out of range";
        return PTG_ERR_INVALID;
      }
    }
  }
  if (bricks) {
    GrainRec& fg = grains[fill];
    int32_t src = 0;
    for (int ig = 1; ig <= m->ngrain; ++ig) {
      for (const Surf& sj : grains[ig].s) {
        const int32_t mpos_j = src++;
        if (!sj.internal) continue;
        Surf s;
        s.gin = fill;
        s.mat1 = 1;
        s.mat2 = sj.mat1;
        s.shape = sj.shape;
        for (int d = 0; d < 3; ++d) s.center[d] = sj.center[d];
        s.radius = sj.radius;
        s.nvertex = sj.nvertex;
        if (s.shape == PTG_SHAPE_POLYGON && s.nvertex > 0) {
          const int n = s.nvertex;
          s.v.resize(3 * (n + 1));
          for (int i = 0; i <= n; ++i)
            for (int d = 0; d < 3; ++d) s.v[3 * i + d] = sj.v[3 * (n - i) + d];
          polygon_setup(s);
        } else if (s.shape == PTG_SHAPE_CAPPED) {
          s.v = sj.v;  /* the same axis: one cylinder seen from the matrix */
        }
        s.gout = sj.gin;
        if (!table_ok(m, s.mat2, s.mat1)) { *why = "transmission table index out of range"; return PTG_ERR_INVALID; }
        interface_props(m, s);
        if (m->surf_spec) s.spec = m->surf_spec[mpos_j];
        fg.s.push_back(s);
      }
    }
    /* periodic faces may not cut a brick: a wrapped phonon keeps its grain */
    for (int f = 2; f < 6; f += 2) {
      if (m->face_kind[f] != PTG_FACE_PERIODIC) continue;
      const int ax = f >> 1;
      for (int ig = 1; ig <= m->ngrain; ++ig) {
        for (const Surf& s : grains[ig].s) {
          if (!s.internal) continue;
          if (s.shape == PTG_SHAPE_POLYGON) {
            for (int i = 0; i < s.nvertex; ++i) {
              double x = s.v[3 * i + ax];
              if (!(x > 0.0 && x < m->box[ax])) { *why = "a brick touches a periodic face"; return PTG_ERR_INVALID; }
            }
          } else if (s.shape == PTG_SHAPE_CAPPED) {
            /* extent of the capped cylinder along this axis */
            const double a = s.v[3 + ax] - s.v[ax];
            double l2 = 0.0;
            for (int d = 0; d < 3; ++d) l2 += (s.v[3 + d] - s.v[d]) * (s.v[3 + d] - s.v[d]);
            const double ca = fabs(a) / sqrt(l2);
            const double ext = 0.5 * fabs(a) + s.radius * sqrt(std::max(0.0, 1.0 - ca * ca));
            const double c = s.center[ax];
            if (!(c - ext > 0.0 && c + ext < m->box[ax])) { *why = "a brick touches a periodic face"; return PTG_ERR_INVALID; }
          } else if (!(s.shape == PTG_SHAPE_CYLINDER && ax == 2)) {
            double c = s.center[ax];
            if (!(c - s.radius > 0.0 && c + s.radius < m->box[ax])) { *why = "a brick touches a periodic face"; return PTG_ERR_INVALID; }
          } else {
            *why = "z-cylinders cannot be cut by periodic z faces";
            return PTG_ERR_INVALID;
          }
        }
      }
    }
  } else {
    for (int f = 2; f < 6; ++f)
      if (m->face_kind[f] == PTG_FACE_PERIODIC) { *why = "periodic faces need bricks"; return PTG_ERR_INVALID; }
  }
  out->shape.clear();
  *out = GeomSoA();
  for (int d = 0; d < 3; ++d) out->box[d] = m->box[d];
  out->scope[0] = m->scope[0];
  out->scope[1] = m->scope[1];
  for (int f = 0; f < 6; ++f) out->face_kind[f] = m->face_kind[f];
  out->kind_grain = m->kind_grain;
  out->ngrain = m->ngrain;
  out->igrain_fill = fill;
  out->nmaterial = m->nmaterial;
  flatten(grains, out);
  return PTG_OK;
}

int copy_geometry(const ptg_geometry* g, GeomSoA* out, std::string* why) {
  if (!g) { *why = "null geometry"; return PTG_ERR_INVALID; }
  if (g->ngrain < 1 || g->ngrain_total < 2 || g->nsurf < 6 || !g->grain_begin || !g->shape) {
    *why = "geometry needs the box grain and >= 1 grain";
    return PTG_ERR_INVALID;
  }
  const int bricks = g->kind_grain == PTG_GRAIN_BRICKS;
  if (g->ngrain_total != g->ngrain + 1 + bricks) { *why = "ngrain_total inconsistent"; return PTG_ERR_INVALID; }
  if (bricks && g->igrain_fill != g->ngrain + 1) { *why = "igrain_fill must be ngrain+1"; return PTG_ERR_INVALID; }
  if (g->grain_begin[0] != 0 || g->grain_begin[1] != 6 || g->grain_begin[g->ngrain_total] != g->nsurf) {
    *why = "grain_begin inconsistent (box grain must hold 6 surfaces)";
    return PTG_ERR_INVALID;
  }
  for (int i = 0; i < g->ngrain_total; ++i)
    if (g->grain_begin[i + 1] < g->grain_begin[i]) { *why = "grain_begin not ascending"; return PTG_ERR_INVALID; }
  for (int d = 0; d < 3; ++d)
    if (!(g->box[d] > 0.0)) { *why = "box lengths must be > 0"; return PTG_ERR_INVALID; }
  *out = GeomSoA();
  for (int d = 0; d < 3; ++d) out->box[d] = g->box[d];
  out->scope[0] = g->scope[0];
  out->scope[1] = g->scope[1];
  for (int f = 0; f < 6; ++f) out->face_kind[f] = g->face_kind[f];
  out->kind_grain = g->kind_grain;
  out->ngrain = g->ngrain;
  out->igrain_fill = g->igrain_fill;
  out->nmaterial = g->nmaterial;
  const int ns = g->nsurf, ngt = g->ngrain_total, nvt = g->nvertex_total;
  out->grain_begin.assign(g->grain_begin, g->grain_begin + ngt + 1);
  out->grain_incident.assign(g->grain_incident, g->grain_incident + ngt);
  out->grain_generatrix.assign(g->grain_generatrix, g->grain_generatrix + 3 * ngt);
  out->shape.assign(g->shape, g->shape + ns);
  out->nvertex.assign(g->nvertex, g->nvertex + ns);
  out->vertex_begin.assign(g->vertex_begin, g->vertex_begin + ns);
  out->vertex.assign(g->vertex, g->vertex + 3 * (size_t)nvt);
  out->normal.assign(g->normal, g->normal + 3 * ns);
  out->tangent.assign(g->tangent, g->tangent + 9 * ns);
  out->center.assign(g->center, g->center + 3 * ns);
  out->radius.assign(g->radius, g->radius + ns);
  out->kind_trans.assign(g->kind_trans, g->kind_trans + ns);
  out->specularity.assign(g->specularity, g->specularity + ns);
  out->trans_param.assign(g->trans_param, g->trans_param + ns);
  out->grain_inside.assign(g->grain_inside, g->grain_inside + ns);
  out->grain_outside.assign(g->grain_outside, g->grain_outside + ns);
  out->internal.assign(g->internal, g->internal + ns);
  out->incident.assign(g->incident, g->incident + ns);
  out->material1.assign(g->material1, g->material1 + ns);
  out->material2.assign(g->material2, g->material2 + ns);
  for (int k = 0; k < ns; ++k) {
    const int sh = out->shape[k];
    if (sh < PTG_SHAPE_POLYGON || sh > PTG_SHAPE_CAPPED) { *why = "unknown surface shape"; return PTG_ERR_INVALID; }
    if (sh == PTG_SHAPE_CAPPED) {
      if (out->nvertex[k] != 2 || out->vertex_begin[k] < 0 || out->vertex_begin[k] + 3 > nvt ||
          !(out->radius[k] > 0.0)) {
        *why = "capped cylinder needs 2 axis end points and a radius > 0";
        return PTG_ERR_INVALID;
      }
      const double* v = &out->vertex[3 * (size_t)out->vertex_begin[k]];
      double l2 = 0.0;
      for (int d = 0; d < 3; ++d) l2 += (v[3 + d] - v[d]) * (v[3 + d] - v[d]);
      if (!(l2 > 0.0)) { *why = "capped cylinder axis must be > 0"; return PTG_ERR_INVALID; }
    } else if (sh == PTG_SHAPE_POLYGON) {
      if (out->nvertex[k] < 3 || out->vertex_begin[k] < 0 ||
          out->vertex_begin[k] + out->nvertex[k] + 1 > nvt) {
        *why = "polygon vertex range out of bounds";
        return PTG_ERR_INVALID;
      }
    } else if (!(out->radius[k] > 0.0)) {
      *why = "sphere/cylinder radius must be > 0";
      return PTG_ERR_INVALID;
    }
    if (out->internal[k] && (out->grain_outside[k] < 0 || out->grain_outside[k] >= ngt)) {
      *why = "grain_outside out of range";
      return PTG_ERR_INVALID;
    }
  }
  out->make_view();
  return PTG_OK;
}

int copy_spectrum(const ptg_spectrum* s, SpecSoA* out, std::string* why) {
  if (!s || s->nbranch < 1 || s->nkpoint < 1 || !s->omega || !s->tau || !s->vel || !s->weight) {
    *why = "spectrum needs nbranch, nkpoint >= 1 and omega/tau/vel/weight";
    return PTG_ERR_INVALID;
  }
  const size_t n = (size_t)s->nbranch * s->nkpoint;
  out->nb = s->nbranch;
  out->nk = s->nkpoint;
  out->rtemp = s->rtemp;
  out->vol = s->vol;
  out->omega.assign(s->omega, s->omega + n);
  out->tau.assign(s->tau, s->tau + n);
  out->vel.assign(s->vel, s->vel + n);
  out->weight.assign(s->weight, s->weight + n);
  if (s->mfp) out->mfp.assign(s->mfp, s->mfp + n); else out->mfp.assign(n, 0.0);
  double mx = out->omega[0];
  for (size_t i = 1; i < n; ++i) if (out->omega[i] > mx) mx = out->omega[i];
  out->max_omega = mx;
  for (size_t i = 0; i < n; ++i) {
    if (!isfinite(out->omega[i]) || !isfinite(out->tau[i]) || !isfinite(out->vel[i])) {
      *why = "non-finite spectrum entry";
      return PTG_ERR_INVALID;
    }
  }
  return PTG_OK;
}

/* ---- ptg_run numbering ------------------------------------------------- */

int64_t run_ntask(const SpecSoA& s, const ptg_run* r) {
  int64_t ns = (r->kind_mfp == PTG_MFP_GRID) ? r->nmfp : 1;
  return (int64_t)s.nb * s.nk * ns * (r->nangle - 1);
}

bool run_valid(const SpecSoA& s, const ptg_run* r, std::string* why) {
  if (!r) { *why = "null run"; return false; }
  if (r->nangle < 3 || (r->nangle % 2) == 0) { *why = "nangle must be odd and >= 3 (Simpson's rule)"; return false; }
  if (r->np < 1) { *why = "np must be >= 1"; return false; }
  if (r->nranks < 1 || r->rank < 0 || r->rank >= r->nranks) { *why = "rank out of range"; return false; }
  if (r->kind_mfp < PTG_MFP_MATTHIESSEN || r->kind_mfp > PTG_MFP_PER_MODE) { *why = "unknown kind_mfp"; return false; }
  if (r->kind_mfp == PTG_MFP_GRID) {
    if (r->nmfp < 1 || !r->mfp_grid_nm) { *why = "GRID needs nmfp >= 1 and the grid"; return false; }
    for (int i = 0; i < r->nmfp; ++i) {
      if (!(r->mfp_grid_nm[i] > 0.0)) { *why = "grid MFPs must be > 0"; return false; }
      if (i > 0 && !(r->mfp_grid_nm[i] > r->mfp_grid_nm[i - 1])) { *why = "grid must ascend"; return false; }
    }
  }
  if (r->kind_mfp != PTG_MFP_MATTHIESSEN && !(r->temperature > 0.0)) { *why = "temperature must be > 0"; return false; }
  if (r->stream < 0 || r->stream >= (1 << 24)) { *why = "stream must be in [0, 2^24)"; return false; }
  if (r->nbins < 0) { *why = "nbins must be >= 0"; return false; }
  if (s.nb < 1) { *why = "no spectrum"; return false; }
  (void)s;
  return true;
}

void run_tasks(const SpecSoA& s, const ptg_run* r, std::vector<TaskHost>* tasks) {
  const int64_t nm = (int64_t)s.nb * s.nk;
  const int64_t ns = (r->kind_mfp == PTG_MFP_GRID) ? r->nmfp : 1;
  const int64_t nt = run_ntask(s, r);
  const double half_pi = 3.14159265358979323846 * 0.5;
  const double scale = (r->scatter_scale > 0.0) ? r->scatter_scale : 1.0;
  /* the angle's cos / sin and the (mode, grid point) MFP, each computed once */
  std::vector<double> ca(r->nangle), sa(r->nangle), lam((size_t)(nm * ns));
  for (int ia = 0; ia < r->nangle; ++ia) {
    const double theta = 0.0 + (double)ia / (double)(r->nangle - 1) * half_pi;
    ca[ia] = cos(theta);
    sa[ia] = sin(theta);
  }
  for (int64_t sg = 0; sg < ns; ++sg)
    for (int64_t m = 0; m < nm; ++m) {
      double l;
      if (r->kind_mfp == PTG_MFP_MATTHIESSEN) {
        l = 1.0e10;
      } else if (r->kind_mfp == PTG_MFP_GRID) {
        l = r->mfp_grid_nm[sg];   /* grid points are sampling points */
      } else {
        const double tau_s = s.tau[m] * 1.0e-12 * (s.rtemp / r->temperature);
        l = tau_s * s.vel[m] * 1.0e9 / scale;
      }
      lam[(size_t)(m + nm * sg)] = l;
    }
  tasks->resize(nt);
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t m = t % nm, rest = t / nm, sg = rest % ns, ia = rest / ns;
    TaskHost& th = (*tasks)[t];
    th.cth = ca[ia];
    th.sth = sa[ia];
    th.omega = s.omega[m];
    th.lambda = lam[(size_t)(m + nm * sg)];
  }
}

void simpson_weights(int na, double box_x, std::vector<double>* coef, double* dS) {
  const double half_pi = 3.14159265358979323846 * 0.5;
  std::vector<double> vangle(na);
  for (int ia = 0; ia < na; ++ia) vangle[ia] = 0.0 + (double)ia / (double)(na - 1) * half_pi;
  *dS = (vangle[1] - vangle[0]) / 3.0 * 3.0 * 0.5 * box_x;
  coef->assign(na, 0.0);
  std::vector<double> ca(na, 0.0);
  for (int ia = 1; ia < na - 1; ia += 2) { ca[ia - 1] += 1.0; ca[ia] += 4.0; ca[ia + 1] += 1.0; }
  for (int ia = 0; ia < na; ++ia) (*coef)[ia] = ca[ia] * (sin(vangle[ia]) * cos(vangle[ia]));
}

void mode_constants(const SpecSoA& s, const ptg_run* r, ModeConst* mc) {
  const double HBAR = 1.054571e-34, KB = 1.3806503e-23;
  const int nm = s.nmode();
  double wsum = 0.0;
  for (int m = 0; m < nm; ++m) wsum += s.weight[m];
  const int nqfbz = (int)(wsum / s.nb);
  mc->K.resize(nm);
  mc->W.resize(nm);
  mc->mfp_m.resize(nm);
  mc->bin.assign(nm, -1);
  const double T = r->temperature;
  for (int m = 0; m < nm; ++m) {
    const double x = HBAR * s.omega[m] / (KB * T);
    double cap;
    if (x <= 1.0e-10) cap = KB;
    else { double q = (x / 2) / sinh(x / 2); cap = KB * (q * q); }
    const double tau = s.tau[m] * 1.0e-12 * (s.rtemp / T);
    const double scale = (r->scatter_scale > 0.0) ? r->scatter_scale : 1.0;
    mc->mfp_m[m] = tau * s.vel[m] / scale;
    mc->K[m] = cap * s.weight[m] * s.vel[m] / 3 / s.vol / nqfbz;
    mc->W[m] = cap * s.weight[m] * s.vel[m];
    if (r->nbins > 0) {
      const double lo = r->bin_omega_min, hi = r->bin_omega_max;
      if (hi > lo && s.omega[m] >= lo && s.omega[m] <= hi) {
        int b = (int)floor((s.omega[m] - lo) / (hi - lo) * r->nbins);
        if (b >= r->nbins) b = r->nbins - 1;
        if (b < 0) b = 0;
        mc->bin[m] = b;
      }
    }
  }
}

}  // namespace ptg

/* ---- C ABI: geometry buffers ------------------------------------------- */

struct ptg_geombuf {
  ptg::GeomSoA g;
};

extern "C" int ptg_geometry_build(const ptg_model* model, const ptg_spectrum* spec,
                                  ptg_geombuf** out) {
  ptg_geombuf* b = nullptr;
  try {
    (void)spec;
    if (!out) return PTG_ERR_INVALID;
    *out = nullptr;
    b = ptg::alloc_should_fail() ? nullptr : new (std::nothrow) ptg_geombuf();
    if (!b) return PTG_ERR_NOMEM;
    std::string why;
    int st = ptg::build_geometry(model, &b->g, &why);
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

extern "C" const ptg_geometry* ptg_geombuf_view(const ptg_geombuf* buf) {
  return buf ? &buf->g.view : nullptr;
}

extern "C" void ptg_geombuf_free(ptg_geombuf* buf) { delete buf; }
