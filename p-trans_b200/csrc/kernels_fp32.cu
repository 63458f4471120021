/*
 * kernels_fp32.cu - persistent FP32 transport kernel.
 *
 * Same physics and random-number counters as the reference's calcTransmit
 * (src/RTMCphon.f90:1608-2414), restructured for the GPU:
 *   - one resident grid; every warp pulls work chunks (task, particle range)
 *     from an atomic queue ordered longest-expected-trajectory first, and a
 *     lane whose phonon has left the box is refilled at once from the warp's
 *     chunk (ballot + popc ranking), so warps stay full while trajectory
 *     lengths differ by orders of magnitude;
 *   - phonon state lives in registers for the whole trajectory;
 *   - geometry (surface records, polygon edge planes, per-grain candidate
 *     lists) is one blob copied into shared memory by a bulk asynchronous copy
 *     when it fits, else read through the read-only path;
 *   - the box grain is an axis-aligned slab test (its six faces are the
 *     reference's box quads, src/RTMCphon.f90:1253-1332);
 *   - intersection is FP32 with an absolute tolerance eps: planes accept
 *     t >= -eps and edge planes accept points within eps, so neighbouring
 *     facets overlap and no ray leaks through a shared edge; quadrics use the
 *     stable quadratic roots, the far root from the inside, and exclude the
 *     surface just left from the outside, which replaces the reference's
 *     absolute 1e-7 nm nudge (src/RTMCphon.f90:1779);
 *   - safe-ball fast path: after an intrinsic (p-p) event a lane with a short
 *     MFP computes a lower bound d of the distance from that point to every
 *     surface of its grain and of the box; while the end point of the next
 *     free path stays inside the ball of radius d around that point the whole
 *     segment does (the ball is convex), so the flight must end in another p-p
 *     event and is taken without an intersection test.  The flight is still
 *     counted and still draws its own Philox block, so the trajectory is the
 *     one the full test gives.  A diffusive walk leaves the ball only after
 *     about (d/MFP)^2 flights, which shortens the serial chain of the longest
 *     trajectories that bound the kernel's run time.  A warp takes fast
 *     flights in groups of four, past fast_steps only while half its live
 *     lanes are still in their balls, so lanes that need a full flight are
 *     not held back.  With the ball the lane keeps a second radius about the
 *     same centre, over the grain's candidate surfaces alone (the grain
 *     ball): a flight inside it needs only the box-face test;
 *   - one Philox4x32-10 block per free flight supplies the four uniforms of
 *     any event; on the fast path the blocks of four flights are computed
 *     together so that four independent chains fill the issue slots; tallies
 *     are integer, aggregated per warp by task (match_any) before one atomic;
 *   - two phases: the drain phase runs the work queue one lane per phonon
 *     and, once the queue is dry, hands its live phonons to a tail list;
 *     the tail phase (a second launch of the same kernel) gives each of them
 *     a warp that advances it 32 flights per round, one flight per lane, with
 *     the flights' start points summed in flight order (in grains with a BVH
 *     a round tests at most kTestWindow flights from its first one outside
 *     the safe ball), and takes the phonon's surface events in the warp too;
 *     every path (fast, full, cooperative) moves the position with the same
 *     fma and takes events with the same code, so a trajectory is the same
 *     whichever path takes its flights.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <type_traits>

#include "kernels.h"
#include "philox.cuh"

namespace ptg {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kBlock = 256;
constexpr float kTwoPi = 6.28318530717958648f;
constexpr float kPi = 3.14159265358979323846f;

extern __shared__ float4 sblob[];

#ifdef PT_CHECK
/* Bounds-checked build: [0] violations, [1] code of the first, [2] its
   index.  A failed check is recorded and the access is redirected to a
   valid element; the kernel never traps. */
__device__ int g_check[3];
__device__ __noinline__ void check_fail(int code, int index) {
  if (atomicAdd(&g_check[0], 1) == 0) {
    g_check[1] = code;
    g_check[2] = index;
  }
}
#endif

/* Geometry blob accessor: SMEM = true reads the copy staged in shared
   memory (shared-memory loads), false reads global memory through the
   read-only path. */
template <bool SMEM>
struct Geo {
  const float4* base;   /* global blob (SMEM = false) */
  BlobLayout lay;
  int nstage = 0;       /* SMEM = false: BVH node units staged in shared memory */
  __device__ __forceinline__ float4 ld(int i) const {
#ifdef PT_CHECK
    if ((unsigned)i >= (unsigned)lay.total) { check_fail(1, i); i = 0; }
#endif
    if (SMEM) return sblob[i];
    return __ldg(base + i);
  }
  __device__ __forceinline__ int ldi(int unit, int k) const {
#ifdef PT_CHECK
    if (k < 0 || (unsigned)(unit + k / 4) >= (unsigned)lay.total) { check_fail(1, unit + k / 4); unit = 0; k = 0; }
#endif
    if (SMEM) return reinterpret_cast<const int*>(sblob + unit)[k];
    return __ldg(reinterpret_cast<const int*>(base + unit) + k);
  }
  __device__ __forceinline__ float4 hotA(int s) const { return ld(lay.hot + 2 * s); }
  __device__ __forceinline__ int4 hotB(int s) const {
    const float4 v = ld(lay.hot + 2 * s + 1);
    return make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z),
                     __float_as_int(v.w));
  }
  __device__ __forceinline__ float4 cold(int s, int i) const { return ld(lay.cold + 3 * s + i); }
  __device__ __forceinline__ float4 edge(int e) const { return ld(lay.edge + e); }
  __device__ __forceinline__ int cand_begin(int g) const { return ldi(lay.cand_begin, g); }
  __device__ __forceinline__ int cand(int k) const { return ldi(lay.cand, k); }
  __device__ __forceinline__ float4 start(int i) const { return ld(lay.start + i); }
  __device__ __forceinline__ int bvh_root(int g) const { return ldi(lay.bvh_root, g); }
  __device__ __forceinline__ float4 node(int i) const {
    if (!SMEM && i < nstage) return sblob[i];  /* a top level, staged */
    return ld(lay.bvh_node + i);
  }
};

/* Square root from the hardware approximation (relative error ~2^-22). */
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

/* sin / cos of 2*pi*u, u in (0,1): hardware approximations on [-pi, pi). */
__device__ __forceinline__ void sincos2pi(float u, float* s, float* c) {
  const float a = fmaf(u, kTwoPi, -kPi);
  *s = -__sinf(a);
  *c = -__cosf(a);
}

/* Geometry accessor of a batched launch: each lane reads the blob of its own
   geometry from global memory. */
struct GeoBatch {
  const float4* base;
  BlobLayout lay;
  int nstage = 0;       /* unused: a batched launch stages nothing */
  __device__ __forceinline__ float4 ld(int i) const {
#ifdef PT_CHECK
    if ((unsigned)i >= (unsigned)lay.total) { check_fail(1, i); i = 0; }
#endif
    return __ldg(base + i);
  }
  __device__ __forceinline__ int ldi(int unit, int k) const {
#ifdef PT_CHECK
    if (k < 0 || (unsigned)(unit + k / 4) >= (unsigned)lay.total) { check_fail(1, unit + k / 4); unit = 0; k = 0; }
#endif
    return __ldg(reinterpret_cast<const int*>(base + unit) + k);
  }
  __device__ __forceinline__ float4 hotA(int s) const { return ld(lay.hot + 2 * s); }
  __device__ __forceinline__ int4 hotB(int s) const {
    const float4 v = ld(lay.hot + 2 * s + 1);
    return make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z),
                     __float_as_int(v.w));
  }
  __device__ __forceinline__ float4 cold(int s, int i) const { return ld(lay.cold + 3 * s + i); }
  __device__ __forceinline__ float4 edge(int e) const { return ld(lay.edge + e); }
  __device__ __forceinline__ int cand_begin(int g) const { return ldi(lay.cand_begin, g); }
  __device__ __forceinline__ int cand(int k) const { return ldi(lay.cand, k); }
  __device__ __forceinline__ float4 start(int i) const { return ld(lay.start + i); }
  __device__ __forceinline__ int bvh_root(int g) const { return ldi(lay.bvh_root, g); }
  __device__ __forceinline__ float4 node(int i) const { return ld(lay.bvh_node + i); }
};

/* Point (x, y, z) on a polygon's plane against its edge half-spaces m
   (unit normal in the plane, pointing in, offset m.w), within eps. */
__device__ __forceinline__ bool inside_edge(float4 m, float x, float y, float z, float eps) {
  return !(fmaf(m.x, x, fmaf(m.y, y, m.z * z)) < m.w - eps);
}

template <class G_t>
__device__ __forceinline__ bool inside_edges(const G_t& G, int e0, int ne, float x, float y,
                                             float z, float eps) {
  for (int e = 0; e < ne; ++e)
    if (!inside_edge(G.edge(e0 + e), x, y, z, eps)) return false;
  return true;
}

/* Candidate order does not change the nearest hit: the raw distance t
   decides and equal distances go to the lower surface index, so a BVH and
   the linear scan of the same grain find the same surface. */
__device__ __forceinline__ bool closer(float t, int s, float tr, int sr) {
  return t < tr || (t == tr && s < sr);
}

/* Polygon s with plane A (unit normal A.xyz along the side it is hit from,
   offset A.w): the ray's crossing of the plane, in front (within eps) and
   nearer than (tr, sb), and inside the edges; the edges are read only for a
   crossing that passes the rest. */
__device__ __forceinline__ float poly_cross(float4 A, float px, float py, float pz, float dx,
                                            float dy, float dz, float eps) {
  /* the plane crossing, or -inf for a ray not heading into the plane's
     front or crossing it behind the start (beyond eps) */
  const float cosa = fmaf(A.x, dx, fmaf(A.y, dy, A.z * dz));
  const float t = __fdividef(A.w - fmaf(A.x, px, fmaf(A.y, py, A.z * pz)), cosa);
  return (cosa > 0.0f && t >= -eps) ? t : -3.0e38f;
}

/* The rest of the polygon test for a plane crossing t (poly_cross): nearer
   than (tr, sb) and inside the edges. */
template <class G_t>
__device__ __forceinline__ void poly_inside(const G_t& G, int s, float t, float px, float py,
                                            float pz, float dx, float dy, float dz, float eps,
                                            float& tr, int& sb) {
  if (!(t >= -eps) || !closer(t, s, tr, sb)) return;
  const int4 B = G.hotB(s);
  const float hx = fmaf(t, dx, px), hy = fmaf(t, dy, py), hz = fmaf(t, dz, pz);
  if (!inside_edges(G, B.y, B.z, hx, hy, hz, eps)) return;
  tr = t;
  sb = s;
}

/* poly_inside for a triangle whose three edges are at E (shared memory). */
__device__ __forceinline__ void tri_inside(const float4* E, int s, float t, float px, float py,
                                           float pz, float dx, float dy, float dz, float eps,
                                           float& tr, int& sb) {
  if (!(t >= -eps) || !closer(t, s, tr, sb)) return;
  const float hx = fmaf(t, dx, px), hy = fmaf(t, dy, py), hz = fmaf(t, dz, pz);
  if (!inside_edge(E[0], hx, hy, hz, eps) || !inside_edge(E[1], hx, hy, hz, eps) ||
      !inside_edge(E[2], hx, hy, hz, eps))
    return;
  tr = t;
  sb = s;
}

template <class G_t>
__device__ __forceinline__ void poly_test(const G_t& G, int s, float4 A, float px, float py,
                                          float pz, float dx, float dy, float dz, float eps,
                                          float& tr, int& sb) {
  poly_inside(G, s, poly_cross(A, px, py, pz, dx, dy, dz, eps), px, py, pz, dx, dy, dz, eps, tr,
              sb);
}

/* Capped cylinder (centre A.xyz, radius A.w; unit axis E.xyz, half length
   E.w) against the ray p + t d.  From inside (interior record) the exit:
   the mantle's far root when its axial coordinate lies within the caps, or
   the cap the ray leaves through when the crossing lies within the radius.
   From outside the entry: the mantle's near root (approaching) within the
   caps, or the cap facing the ray within the radius; the cylinder just left
   is excluded, as for the other quadrics.  Tolerance eps on both limits. */
template <class G_t>
__device__ __forceinline__ void capped_test(const G_t& G, int s, float4 A, int4 B, float px,
                                            float py, float pz, float dx, float dy, float dz,
                                            int last_geom, float eps, float& tr, int& sb) {
  const bool interior = (B.x & REC_INTERIOR) != 0;
  if (!interior && B.w == last_geom) return;
  const float4 E = G.edge(B.y);
  const float wx = A.x - px, wy = A.y - py, wz = A.z - pz;   /* centre - p */
  const float sw = fmaf(wx, E.x, fmaf(wy, E.y, wz * E.z));
  const float s0 = -sw;                                      /* axial coordinate of p */
  const float ds = fmaf(dx, E.x, fmaf(dy, E.y, dz * E.z));
  const float upx = fmaf(-sw, E.x, wx), upy = fmaf(-sw, E.y, wy), upz = fmaf(-sw, E.z, wz);
  const float vpx = fmaf(-ds, E.x, dx), vpy = fmaf(-ds, E.y, dy), vpz = fmaf(-ds, E.z, dz);
  const float a = fmaf(vpx, vpx, fmaf(vpy, vpy, vpz * vpz));
  const float b = fmaf(upx, vpx, fmaf(upy, vpy, upz * vpz));
  const float c = fmaf(upx, upx, fmaf(upy, upy, upz * upz)) - A.w * A.w;
  const float hl = E.w + eps, rr = (A.w + eps) * (A.w + eps);
  float t = 3.0e38f;
  /* mantle: roots of a t^2 - 2 b t + c = 0 */
  if (a > 0.0f) {
    const float disc = fmaf(b, b, -a * c);
    if (disc >= 0.0f) {
      const float sq = sqrtf(disc);
      float tl = 3.0e38f;
      if (interior) tl = (b >= 0.0f) ? __fdividef(b + sq, a) : __fdividef(-c, sq - b);
      else if (b > 0.0f) tl = __fdividef(c, b + sq);
      if (tl >= -eps && fabsf(fmaf(tl, ds, s0)) <= hl) t = tl;
    }
  }
  /* caps */
  if (ds != 0.0f) {
    float tc;
    if (interior) tc = __fdividef((ds > 0.0f ? E.w : -E.w) - s0, ds);
    else if (s0 < -E.w && ds > 0.0f) tc = __fdividef(-E.w - s0, ds);
    else if (s0 > E.w && ds < 0.0f) tc = __fdividef(E.w - s0, ds);
    else tc = 3.0e38f;
    if (tc >= -eps && tc < t) {
      const float qx = fmaf(-tc, vpx, upx), qy = fmaf(-tc, vpy, upy), qz = fmaf(-tc, vpz, upz);
      if (fmaf(qx, qx, fmaf(qy, qy, qz * qz)) <= rr) t = tc;
    }
  }
  if (!(t < 3.0e38f) || !closer(t, s, tr, sb)) return;
  tr = t;
  sb = s;
}

/* Outward normal of the capped-cylinder piece nearer to p: a cap (+-axis)
   when the axial distance to it is the smaller, else the mantle's radial
   direction. */
__device__ __forceinline__ void capped_normal(float4 A, float4 E, float px, float py, float pz,
                                              float& nx, float& ny, float& nz) {
  const float wx = px - A.x, wy = py - A.y, wz = pz - A.z;
  const float sa = fmaf(wx, E.x, fmaf(wy, E.y, wz * E.z));
  const float ux = fmaf(-sa, E.x, wx), uy = fmaf(-sa, E.y, wy), uz = fmaf(-sa, E.z, wz);
  const float rho = sqrtf(fmaf(ux, ux, fmaf(uy, uy, uz * uz)));
  if (fabsf(fabsf(sa) - E.w) < fabsf(rho - A.w)) {
    const float sg = sa < 0.0f ? -1.0f : 1.0f;
    nx = sg * E.x; ny = sg * E.y; nz = sg * E.z;
  } else {
    const float inv = __frcp_rn(rho);
    nx = ux * inv; ny = uy * inv; nz = uz * inv;
  }
}

/* One candidate surface against the ray p + t d: updates the nearest raw
   distance tr and surface sb. */
template <bool EXT, class G_t>
__device__ __forceinline__ void test_surface(const G_t& G, int s, float px, float py, float pz,
                                             float dx, float dy, float dz, int last_geom,
                                             float eps, float zmax, float& tr, int& sb) {
  const float4 A = G.hotA(s);
  const int4 B = G.hotB(s);
  const int type = B.x & 0xff;
  if (EXT && type == REC_CAP) {
    capped_test(G, s, A, B, px, py, pz, dx, dy, dz, last_geom, eps, tr, sb);
  } else if (type == REC_POLY) {
    poly_test(G, s, A, px, py, pz, dx, dy, dz, eps, tr, sb);
  } else {
    /* sphere or z cylinder, written with selects: the lanes of a warp test
       the same surface with different rays, so the only branch is the one
       around the square root (a ray that misses) */
    const bool interior = (B.x & REC_INTERIOR) != 0;
    const bool sph = type == REC_SPHERE;
    const float wx = A.x - px, wy = A.y - py;
    const float wz = sph ? A.z - pz : 0.0f, ez = sph ? dz : 0.0f;
    const float r = sph ? A.w : A.z;
    const float a = sph ? 1.0f : fmaf(dx, dx, dy * dy);
    const float b = fmaf(wx, dx, fmaf(wy, dy, wz * ez));
    const float c = fmaf(wx, wx, fmaf(wy, wy, wz * wz)) - r * r;
    /* roots of a t^2 - 2 b t + c = 0 */
    const float disc = fmaf(b, b, -a * c);
    if ((interior || B.w != last_geom) && a > 0.0f && disc >= 0.0f) {
      const float sq = sqrtf(disc);
      /* from inside the far root (b + sq)/a, written without cancellation;
         from outside the near root (b - sq)/a = c / (b + sq), valid when
         approaching */
      const bool bp = b >= 0.0f;
      const float num = interior ? (bp ? b + sq : -c) : c;
      const float den = interior ? (bp ? a : sq - b) : b + sq;
      const float t = __fdividef(num, den);
      const float hz = fmaf(t, dz, pz);
      const bool ok = (interior || (b > 0.0f && t >= -eps)) && closer(t, s, tr, sb) &&
                      (type != REC_CYL || !(hz < 0.0f || hz > zmax));
      tr = ok ? t : tr;
      sb = ok ? s : sb;
    }
  }
}

/* Entry distance of the ray into a node box (+inf when it misses the box
   or enters beyond tmax); inverse direction components are finite. */
__device__ __forceinline__ float box_entry(float4 lo, float4 hi, float px, float py, float pz,
                                           float ix, float iy, float iz, float tmax, float eps) {
  const float ax = (lo.x - px) * ix, bx = (hi.x - px) * ix;
  const float ay = (lo.y - py) * iy, by = (hi.y - py) * iy;
  const float az = (lo.z - pz) * iz, bz = (hi.z - pz) * iz;
  const float t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
  const float t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
  return (t0 <= t1 && t1 >= -eps && t0 <= tmax) ? t0 : 3.0e38f;
}

__device__ __forceinline__ float inv_dir(float d) {
  return __fdividef(1.0f, fabsf(d) > 1.0e-20f ? d : copysignf(1.0e-20f, d));
}

/* Traversal depth bound: the builder limits the depth to 30. */
constexpr int kBvhStack = 32;

/* BVH traversal of a grain (root >= 0): ordered descent, the far child
   pushed with its entry distance and popped only while it can still hold a
   nearer hit.  Nodes entered beyond tcut (the flight's free path) are
   skipped as well: a flight only needs every hit up to its free path (a hit
   there ends it; with none, a p-p event ends it), so the decision, and the
   trajectory, are those of the full search.  Kept out of line so the linear
   scan that every small grain uses stays compact in the instruction cache. */
template <bool EXT, class G_t>
__device__ __noinline__ void scan_bvh(const G_t& G, int root, float px, float py, float pz,
                                      float dx, float dy, float dz, int last_geom, float eps,
                                      float zmax, float tcut, float& tr, int& sb, unsigned& nbox,
                                      unsigned& nsurf) {
  const float ix = inv_dir(dx), iy = inv_dir(dy), iz = inv_dir(dz);
  int stk[kBvhStack];
  float stt[kBvhStack];
  int sp = 0;
  int node = root;
  while (true) {
    const float4 n1 = G.node(2 * node + 1);
    const int cnt = __float_as_int(n1.w);
    const int a = __float_as_int(G.node(2 * node).w);
    bool descended = false;
    if (cnt > 0) {
      nsurf += (unsigned)cnt;
      for (int k = a; k < a + cnt; ++k)
        test_surface<EXT>(G, G.cand(k), px, py, pz, dx, dy, dz, last_geom, eps, zmax, tr, sb);
    } else {
      nbox += 2u;
      const float tm = fminf(tr, tcut);
      const float tl = box_entry(G.node(2 * a), G.node(2 * a + 1), px, py, pz, ix, iy, iz, tm, eps);
      const float tg = box_entry(G.node(2 * a + 2), G.node(2 * a + 3), px, py, pz, ix, iy, iz, tm,
                                 eps);
      const bool hl = tl < 3.0e38f, hg = tg < 3.0e38f;
      if (hl && hg) {
        const bool lf = tl <= tg;
        if (sp < kBvhStack) {
          stk[sp] = lf ? a + 1 : a;
          stt[sp] = lf ? tg : tl;
          ++sp;
        }
        node = lf ? a : a + 1;
        descended = true;
      } else if (hl || hg) {
        node = hl ? a : a + 1;
        descended = true;
      }
    }
    if (descended) continue;
    bool found = false;
    while (sp > 0) {
      --sp;
      if (stt[sp] <= fminf(tr, tcut)) {
        node = stk[sp];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
}

/* Nearest surface of a grain: its BVH when it has one (kernels built with
   EXT = true, for structures with a BVH or capped cylinders; the others
   never look for either), else every candidate.  tb
   (the box-grain exit, >= 0) and sb are updated; tb stays >= 0.  fp is the
   flight's free path: a BVH search skips what lies beyond it (a hit farther
   away cannot end the flight). */
template <bool EXT, class G_t>
__device__ __forceinline__ void scan_grain(const G_t& G, int grain, float px, float py, float pz,
                                           float dx, float dy, float dz, int last_geom, float eps,
                                           float zmax, float fp, float& tb, int& sb, unsigned& nbox,
                                           unsigned& nsurf) {
  float tr = tb;
  const int root = EXT ? G.bvh_root(grain) : -1;
  if (root < 0) {
    const int kb = G.cand_begin(grain), ke = G.cand_begin(grain + 1);
    nsurf += (unsigned)(ke - kb);
    for (int k = kb; k < ke; ++k)
      test_surface<EXT>(G, G.cand(k), px, py, pz, dx, dy, dz, last_geom, eps, zmax, tr, sb);
  } else {
    scan_bvh<EXT>(G, root, px, py, pz, dx, dy, dz, last_geom, eps, zmax, fp, tr, sb, nbox, nsurf);
  }
  tb = fmaxf(tr, 0.0f);
}

/* Exit of the box grain along d from p: distance tb and face sb (0 x-,
   1 x+, 2 y-, 3 y+, 4 z-, 5 z+), clamped at 0. */
__device__ __forceinline__ void slab_exit(float px, float py, float pz, float dx, float dy,
                                          float dz, float X, float Y, float Z, float& tb,
                                          int& sb) {
  /* selects, no branches: the lanes of a warp go different ways */
  const float tx = __fdividef(dx > 0.0f ? X - px : -px, dx);
  const float ty = __fdividef((dy > 0.0f ? Y : 0.0f) - py, dy);
  const float tz = __fdividef((dz > 0.0f ? Z : 0.0f) - pz, dz);
  const bool hx = dx > 0.0f || dx < 0.0f;
  tb = hx ? tx : 3.0e38f;
  sb = hx ? (dx > 0.0f ? 1 : 0) : -1;
  const bool hy = dy != 0.0f && ty < tb;
  tb = hy ? ty : tb;
  sb = hy ? (dy > 0.0f ? 3 : 2) : sb;
  const bool hz = dz != 0.0f && tz < tb;
  tb = hz ? tz : tb;
  sb = hz ? (dz > 0.0f ? 5 : 4) : sb;
  tb = fmaxf(tb, 0.0f);
}

/* Lower bound of the distance from p to one candidate surface (planes bound
   polygons from below, the infinite cylinder bounds the clipped one).  The
   square roots are the hardware approximation: its relative error (< 2^-22
   of a distance below the box diagonal) is far inside the 4 eps the callers
   take off, so the bound stays a bound. */
template <bool EXT, class G_t>
__device__ __forceinline__ float surface_lb(const G_t& G, int s, float px, float py, float pz) {
  const float4 A = G.hotA(s);
  const int4 B = G.hotB(s);
  const int type = B.x & 0xff;
  if (type == REC_POLY) return fabsf(A.w - fmaf(A.x, px, fmaf(A.y, py, A.z * pz)));
  if (EXT && type == REC_CAP) {
    /* inside: the nearer of mantle and caps; outside: the larger excess */
    const float4 E = G.edge(B.y);
    const float wx = px - A.x, wy = py - A.y, wz = pz - A.z;
    const float sa = fmaf(wx, E.x, fmaf(wy, E.y, wz * E.z));
    const float ux = fmaf(-sa, E.x, wx), uy = fmaf(-sa, E.y, wy), uz = fmaf(-sa, E.z, wz);
    const float er = sqrt_approx(fmaf(ux, ux, fmaf(uy, uy, uz * uz))) - A.w;
    const float ea = fabsf(sa) - E.w;
    return (er <= 0.0f && ea <= 0.0f) ? fminf(-er, -ea) : fmaxf(er, ea);
  }
  if (type == REC_SPHERE) {
    const float wx = px - A.x, wy = py - A.y, wz = pz - A.z;
    return fabsf(sqrt_approx(fmaf(wx, wx, fmaf(wy, wy, wz * wz))) - A.w);
  }
  const float wx = px - A.x, wy = py - A.y;
  return fabsf(sqrt_approx(fmaf(wx, wx, wy * wy)) - A.z);
}

/* Distance from p to a node box (0 inside; approximate square root, as in
   surface_lb). */
__device__ __forceinline__ float box_dist(float4 lo, float4 hi, float px, float py, float pz) {
  const float ex = fmaxf(fmaxf(lo.x - px, px - hi.x), 0.0f);
  const float ey = fmaxf(fmaxf(lo.y - py, py - hi.y), 0.0f);
  const float ez = fmaxf(fmaxf(lo.z - pz, pz - hi.z), 0.0f);
  return sqrt_approx(fmaf(ex, ex, fmaf(ey, ey, ez * ez)));
}

/* BVH range query for the safe ball: the smallest lower bound d of the
   distance from p to a surface of the grain, the surface it belongs to
   (near) and the smallest bound d2 of every other surface, searched below
   the initial d (nodes no nearer than the second bound so far are pruned:
   they cannot change either; a surface's bound is the larger of the
   distance to its leaf's box and its own plane / quadric bound).  Out of
   line, like scan_bvh. */
template <bool EXT, class G_t>
__device__ __noinline__ float safety_bvh(const G_t& G, int root, float px, float py, float pz,
                                         float d, float& d2, int& near) {
  int stk[kBvhStack];
  float std_[kBvhStack];
  int sp = 0;
  int node = root;
  d2 = d;
  near = -1;
  while (true) {
    const float4 n0 = G.node(2 * node), n1 = G.node(2 * node + 1);
    const int cnt = __float_as_int(n1.w);
    const int a = __float_as_int(n0.w);
    bool descended = false;
    if (cnt > 0) {
      const float bd = box_dist(n0, n1, px, py, pz);
      for (int k = a; k < a + cnt; ++k) {
        const int sk = G.cand(k);
        const float e = fmaxf(bd, surface_lb<EXT>(G, sk, px, py, pz));
        const bool nearer = e < d;
        d2 = nearer ? d : fminf(d2, e);
        near = nearer ? sk : near;
        d = nearer ? e : d;
      }
    } else {
      const float dl = box_dist(G.node(2 * a), G.node(2 * a + 1), px, py, pz);
      const float dg = box_dist(G.node(2 * a + 2), G.node(2 * a + 3), px, py, pz);
      const bool lf = dl <= dg;
      const float dn = lf ? dl : dg, df = lf ? dg : dl;
      if (dn < d2) {
        if (df < d2 && sp < kBvhStack) {
          stk[sp] = lf ? a + 1 : a;
          std_[sp] = df;
          ++sp;
        }
        node = lf ? a : a + 1;
        descended = true;
      }
    }
    if (descended) continue;
    bool found = false;
    while (sp > 0) {
      --sp;
      if (std_[sp] < d2) {
        node = stk[sp];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  return d;
}

/* Lower bound of the distance from p to every box face and to every
   candidate surface of the grain, less 4 eps.  A grain with a BVH is
   searched only within `cap` (the radius the safe ball needs).  dgrain
   receives the bound over the candidate surfaces alone (the grain ball: a
   flight inside it needs the box-face test only); for a BVH grain it is
   searched no farther than the full bound, so it costs no extra nodes. */
template <bool EXT, class G_t>
__device__ __forceinline__ float safety(const G_t& G, int grain, float px, float py, float pz,
                                        float X, float Y, float Z, float eps, float cap,
                                        float& dgrain, float& dgrain2, int& near) {
  const float dbox = fminf(fminf(fminf(px, X - px), fminf(py, Y - py)), fminf(pz, Z - pz));
  float dc = 3.0e38f, dc2 = 3.0e38f;
  near = -1;
  if (grain > 0) {
    const int root = EXT ? G.bvh_root(grain) : -1;
    if (root < 0) {
      /* the nearest candidate and the bound of all the others */
      const int kb = G.cand_begin(grain), ke = G.cand_begin(grain + 1);
      for (int k = kb; k < ke; ++k) {
        const int sk = G.cand(k);
        const float d = surface_lb<EXT>(G, sk, px, py, pz);
        const bool nearer = d < dc;
        dc2 = nearer ? dc : fminf(dc2, d);
        near = nearer ? sk : near;
        dc = nearer ? d : dc;
      }
    } else {
      dc = safety_bvh<EXT>(G, root, px, py, pz, fminf(dbox, cap), dc2, near);
    }
  }
  dgrain = dc - 4.0f * eps;
  dgrain2 = dc2 - 4.0f * eps;
  return fminf(dbox, dc) - 4.0f * eps;
}

/* One candidate surface, where the second ball has shown it to be the only
   one a flight can reach: scan_grain's result for that flight. */
template <bool EXT, class G_t>
__device__ __forceinline__ void test_near(const G_t& G, int s, float px, float py, float pz,
                                          float dx, float dy, float dz, int last_geom, float eps,
                                          float zmax, float& tb, int& sb, unsigned& nsurf) {
  float tr = tb;
  nsurf += 1u;
  test_surface<EXT>(G, s, px, py, pz, dx, dy, dz, last_geom, eps, zmax, tr, sb);
  tb = fmaxf(tr, 0.0f);
}

/* Local candidate list of the tail phase's rounds in a BVH grain: the
   surfaces of one grain whose bound from a centre c is below a radius R,
   at most kList of them, one per lane.  A flight that starts and ends
   within R - 4 eps of c can meet only listed surfaces, and the safe ball of
   a point p within that radius follows from the listed bounds and
   R - |p - c|, so while the walk stays near c neither needs the tree. */
constexpr int kList = 32;
/* radius of a new list, in units of the MFP (the safe ball's cap) */
constexpr float kListMfp = 32.0f;

/* Largest v over the warp and the lowest lane holding it. */
__device__ __forceinline__ void warp_argmax(float v, int lane, float& vmax, int& lmax) {
  int l = lane;
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(FULL, v, o);
    const int ol = __shfl_xor_sync(FULL, l, o);
    const bool other = ov > v || (ov == v && ol < l);
    v = other ? ov : v;
    l = other ? ol : l;
  }
  vmax = v;
  lmax = l;
}

/* BVH range query for a local list: the surfaces of the grain whose bound
   from p (as in safety_bvh) is below R, kList at most: lane k holds entry
   k while the tree is searched; once the list is full a nearer surface
   replaces the one with the largest bound, and R drops to the bound of
   whatever leaves the list.  Returns the final R (every surface missing
   from the list has a bound of at least R from p) and stores the entries
   to lst, their planes (hotA) to lpl and, for triangles, their edges to
   led (three per entry); kind is 2 when every entry is a triangle, 1 when
   every entry is a polygon, else 0.  Warp-collective: every lane searches
   the same nodes. */
template <bool EXT, class G_t>
__device__ __noinline__ float list_bvh(const G_t& G, int root, float px, float py, float pz,
                                       float R, int lane, int* lst, float4* lpl, float4* led,
                                       int& n, int& kind) {
  int stk[kBvhStack];
  float std_[kBvhStack];
  int sp = 0;
  int node = root;
  int my_s = -1;
  float my_e = -1.0f;
  float emax = 3.0e38f;
  int lmax = 0;
  n = 0;
  while (true) {
    const float4 n0 = G.node(2 * node), n1 = G.node(2 * node + 1);
    const int cnt = __float_as_int(n1.w);
    const int a = __float_as_int(n0.w);
    bool descended = false;
    if (cnt > 0) {
      const float bd = box_dist(n0, n1, px, py, pz);
      for (int k = a; k < a + cnt; ++k) {
        const int sk = G.cand(k);
        const float e = fmaxf(bd, surface_lb<EXT>(G, sk, px, py, pz));
        if (e < R) {
          if (n < kList) {
            if (lane == n) { my_s = sk; my_e = e; }
            if (++n == kList) warp_argmax(my_e, lane, emax, lmax);
          } else if (e < emax) {
            R = fminf(R, emax);
            if (lane == lmax) { my_s = sk; my_e = e; }
            warp_argmax(my_e, lane, emax, lmax);
          } else {
            R = e;
          }
        }
      }
    } else {
      const float dl = box_dist(G.node(2 * a), G.node(2 * a + 1), px, py, pz);
      const float dg = box_dist(G.node(2 * a + 2), G.node(2 * a + 3), px, py, pz);
      const bool lf = dl <= dg;
      const float dn = lf ? dl : dg, df = lf ? dg : dl;
      if (dn < R) {
        if (df < R && sp < kBvhStack) {
          stk[sp] = lf ? a + 1 : a;
          std_[sp] = df;
          ++sp;
        }
        node = lf ? a : a + 1;
        descended = true;
      }
    }
    if (descended) continue;
    bool found = false;
    while (sp > 0) {
      --sp;
      if (std_[sp] < R) {
        node = stk[sp];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  bool poly = true, tri = true;
  if (lane < n) {
    lst[lane] = my_s;
    lpl[lane] = G.hotA(my_s);
    const int4 B = G.hotB(my_s);
    poly = (B.x & 0xff) == REC_POLY;
    tri = poly && B.z == 3;
    if (tri) {
      led[3 * lane] = G.edge(B.y);
      led[3 * lane + 1] = G.edge(B.y + 1);
      led[3 * lane + 2] = G.edge(B.y + 2);
    }
  }
  kind = __all_sync(FULL, tri) ? 2 : (__all_sync(FULL, poly) ? 1 : 0);
  return R;
}

/* safety() for a point p within the radius lc.w of a local list's centre
   lc.xyz: the listed surfaces' bounds (lane k takes entry k) and
   lc.w - |p - c| for every other surface of the grain.  Warp-collective. */
template <bool EXT, class G_t>
__device__ __forceinline__ float safety_list(const G_t& G, const int* lst, int n, float4 lc,
                                             float px, float py, float pz, float X, float Y,
                                             float Z, float eps, int lane, float& dgrain,
                                             float& dgrain2, int& near) {
  const float dbox = fminf(fminf(fminf(px, X - px), fminf(py, Y - py)), fminf(pz, Z - pz));
  float e = 3.0e38f, e2 = 3.0e38f;
  int s = -1;
  if (lane < n) {
    s = lst[lane];
    e = surface_lb<EXT>(G, s, px, py, pz);
  }
  /* the smallest bound, its surface and the second smallest */
  for (int o = 16; o > 0; o >>= 1) {
    const float oe = __shfl_xor_sync(FULL, e, o), oe2 = __shfl_xor_sync(FULL, e2, o);
    const int os = __shfl_xor_sync(FULL, s, o);
    const bool other = oe < e || (oe == e && os < s);
    e2 = other ? fminf(e, oe2) : fminf(oe, e2);
    e = other ? oe : e;
    s = other ? os : s;
  }
  const float wx = px - lc.x, wy = py - lc.y, wz = pz - lc.z;
  const float du = lc.w - sqrt_approx(fmaf(wx, wx, fmaf(wy, wy, wz * wz)));
  near = e < du ? s : -1;
  const float dc = fminf(e, du);
  dgrain = dc - 4.0f * eps;
  dgrain2 = (near >= 0 ? fminf(e2, du) : dc) - 4.0f * eps;
  return fminf(dbox, dc) - 4.0f * eps;
}

/* scan_grain over a local list, for a flight within its radius: the listed
   surfaces are the only ones the flight can meet.  A hit beyond the free
   path cannot end the flight, so the search stops at the float above fp:
   the nearest hit up to fp is the full scan's, and without one tb stays
   above fp, as it would. */
template <bool EXT, class G_t>
__device__ __forceinline__ void scan_list(const G_t& G, const int* lst, const float4* lpl,
                                          const float4* led, int n, int kind, float px, float py,
                                          float pz, float dx, float dy, float dz, int last_geom,
                                          float eps, float zmax, float fp, float& tb, int& sb,
                                          unsigned& nsurf) {
  float tr = fminf(tb, __uint_as_float(__float_as_uint(fp) + 1u));
  nsurf += (unsigned)n;
  if (kind == 2) {
    /* triangles: planes and edges from the list's shared-memory copy */
    for (int k = 0; k < n; k += 4) {
      float t[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        t[i] = k + i < n ? poly_cross(lpl[min(k + i, n - 1)], px, py, pz, dx, dy, dz, eps)
                         : -3.0e38f;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (t[i] > -3.0e38f && t[i] <= tr)
          tri_inside(led + 3 * (k + i), lst[k + i], t[i], px, py, pz, dx, dy, dz, eps, tr, sb);
    }
  } else if (kind == 1) {
    /* polygons only: the planes come from the list's shared-memory copy,
       four crossings at a time (independent), then the edges in list
       order only for a crossing in front of the ray and in range */
    for (int k = 0; k < n; k += 4) {
      float t[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        t[i] = k + i < n ? poly_cross(lpl[min(k + i, n - 1)], px, py, pz, dx, dy, dz, eps)
                         : -3.0e38f;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (t[i] > -3.0e38f && t[i] <= tr)
          poly_inside(G, lst[k + i], t[i], px, py, pz, dx, dy, dz, eps, tr, sb);
    }
  } else {
    for (int k = 0; k < n; ++k)
      test_surface<EXT>(G, lst[k], px, py, pz, dx, dy, dz, last_geom, eps, zmax, tr, sb);
  }
  tb = fmaxf(tr, 0.0f);
}

/* Adjoint accumulators of the sample: dlogP/dp of surface k goes to
   base + k, in shared memory (sh) when the block holds them, else global. */
struct AdjAcc {
  double* sh;
  double* gl;
  float w;
  int base;
  bool in_smem;
};

/* The event at the end of a flight that reaches a surface or box face at
   distance tb along its direction (calcTransmit's collision branch,
   src/RTMCphon.f90:1744-1792, with 2225-2413): the phonon moves to the hit
   point and keeps the rest of its free path; the bath faces end it
   (returns 1 for x-, 2 for x+), a periodic face wraps it, and any other
   surface reflects it (determinSpecular, then reflectSpecular or
   reflectDiffusive) or lets it through into the grain on the other side
   (determinTransmit).  Returns -1 while the phonon goes on.  u0..u3 are
   the flight's Philox uniforms.  The one-lane path and the tail phase's
   rounds both take their events here, so a trajectory does not depend on
   which of them met the surface. */
template <int MODE, bool EXT, class G_t>
__device__ __forceinline__ int surface_hit(const G_t& G, float tb, int sb, float u0, float u1,
                                           float u2, float u3, float Y, float Z, int pmask,
                                           int nmat, float omr, float lam, uint32_t flight,
                                           uint32_t c1, uint32_t slo, uint32_t shi, Key2 key,
                                           const AdjAcc& acc, float& px, float& py, float& pz,
                                           float& dx, float& dy, float& dz, float& fp, int& grain,
                                           float& gr2, float& g2r2, int& last_geom) {
  int end_side = -1;
  px = fmaf(tb, dx, px);
  py = fmaf(tb, dy, py);
  pz = fmaf(tb, dz, pz);
  fp -= tb;
  if (sb == 0) {
    end_side = 1;
  } else if (sb == 1) {
    end_side = 2;
  } else if (sb < 6 && ((pmask >> sb) & 1)) {
    const int ax = sb >> 1;
    const float L = ax == 1 ? Y : Z;
    const float sg = (sb & 1) ? -L : L;
    if (ax == 1) py += sg; else pz += sg;
    last_geom = -1;
  } else {
    const float4 C0 = G.cold(sb, 0), C1 = G.cold(sb, 1), C2 = G.cold(sb, 2);
    const int meta = __float_as_int(C2.w);
    const int kind = meta & 0xff;
    /* transmission threshold: a fixed value, or Gamma / TBC of the mode
       (one material) or drawn between the two materials' values */
    float thr = 0.0f;
    if (kind == 1) {
      thr = C1.w;
    } else if (kind == 2 || kind == 3) {
      if (nmat == 1) {
        thr = __frcp_rn(fmaf(C1.w, omr, 1.0f));
      } else {
        const uint4 R2 = philox10(flight, c1 | 1u, slo, shi, key);
        const float t11 = __frcp_rn(C1.w + 1.0f);
        thr = fmaf(u23f(R2.x), 1.0f - t11, t11);
      }
    }
    /* surface normal at the hit point and surface frame */
    float nx, ny, nz, ax1, ay1, az1, ax2, ay2, az2;
    const int4 B = G.hotB(sb);
    const int type = B.x & 0xff;
    if (type == REC_POLY) {
      nx = C2.x; ny = C2.y; nz = C2.z;
      ax1 = C0.x; ay1 = C0.y; az1 = C0.z;
      ax2 = C1.x; ay2 = C1.y; az2 = C1.z;
    } else {
      const float4 A = G.hotA(sb);
      if (EXT && type == REC_CAP) {
        capped_normal(A, G.edge(B.y), px, py, pz, nx, ny, nz);
      } else {
        float rx = px - A.x, ry = py - A.y, rz = (type == REC_SPHERE) ? pz - A.z : 0.0f;
        const float inv = rsqrtf(fmaf(rx, rx, fmaf(ry, ry, rz * rz)));
        nx = rx * inv; ny = ry * inv; nz = rz * inv;
      }
      const float q2 = fmaf(nx, nx, ny * ny);
      if (q2 > 1.0e-12f) {
        const float q = rsqrtf(q2);
        ax2 = -ny * q; ay2 = nx * q; az2 = 0.0f;
        /* t1 = t2 x n */
        ax1 = ay2 * nz - az2 * ny;
        ay1 = az2 * nx - ax2 * nz;
        az1 = ax2 * ny - ay2 * nx;
      } else {
        ax2 = 0.0f; ay2 = 1.0f; az2 = 0.0f;
        ax1 = 1.0f; ay1 = 0.0f; az1 = 0.0f;
      }
    }
    /* tmpNormal oriented along the incoming direction */
    const float dn0 = fmaf(nx, dx, fmaf(ny, dy, nz * dz));
    const float on = dn0 < 0.0f ? -1.0f : 1.0f;
    bool transmitted = false;
    if (MODE == MODE_ADJOINT) {
      /* d log P / d p of the specular (1/p) or diffuse (-1/(1-p)) choice */
      const float pk = C0.w;
      if (pk > 0.0f && pk < 1.0f) {
        const double sc = (u0 <= pk) ? 1.0 / (double)pk : -1.0 / (1.0 - (double)pk);
        const double v = (double)acc.w * sc;
        const int idx = acc.base + sb;
        if (acc.in_smem) atomicAdd(&acc.sh[idx], v);
        else atomicAdd(&acc.gl[idx], v);
      }
    }
    if (u0 <= C0.w) {
      if (u1 <= thr) {
        transmitted = true;
      } else {
        const float k2 = 2.0f * dn0;
        dx = fmaf(-k2, nx, dx);
        dy = fmaf(-k2, ny, dy);
        dz = fmaf(-k2, nz, dz);
        const float inv = rsqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        dx *= inv; dy *= inv; dz *= inv;
      }
    } else {
      const float sint = sqrt_approx(u1);
      const float cost = sqrt_approx(fmaxf(0.0f, 1.0f - u1));
      float sp, cp;
      sincos2pi(u2, &sp, &cp);
      const float a = sint * cp, b = sint * sp;
      const float vx = fmaf(ax1, a, fmaf(ax2, b, nx * cost));
      const float vy = fmaf(ay1, a, fmaf(ay2, b, ny * cost));
      const float vz = fmaf(az1, a, fmaf(az2, b, nz * cost));
      /* Lambertian into the incidence side, then optionally through */
      const float s = on * fmaf(vx, nx, fmaf(vy, ny, vz * nz));
      float sg = s > 0.0f ? -1.0f : 1.0f;
      if (u3 <= thr) { sg = -sg; transmitted = true; }
      dx = sg * vx; dy = sg * vy; dz = sg * vz;
    }
    if (transmitted) {
      grain = meta >> 8;
      gr2 = 0.0f;
      g2r2 = 0.0f;
    }
    last_geom = B.w;
  }
  /* a free path used up at the surface: a new one */
  if (end_side < 0 && fp < 1.0e-10f) {
    const uint4 R2 = philox10(flight, c1 | 1u, slo, shi, key);
    fp = -lam * __logf(u23f(R2.y));
  }
  return end_side;
}

/* Trace replay: position after flight f of the sample in replay-list slot t
   (f = 0: the emission point), when the host gave a position buffer. */
__device__ __forceinline__ void trace_put(const RunF32& r, long long t, unsigned f, float px,
                                          float py, float pz) {
  if (!r.trace) return;
  const long long at = r.trace_off[t] + f;
  if (at >= r.trace_off[t + 1]) return;
  r.trace[3 * at] = px;
  r.trace[3 * at + 1] = py;
  r.trace[3 * at + 2] = pz;
}

/* The Philox blocks of flights f+1+s+lane, s in [0, 32], from those of
   f+1+lane (cur) and f+33+lane (nxt) held across the warp: a round that
   advances s flights passes the blocks it drew on instead of drawing them
   again (the blocks depend on the flight counter alone). */
__device__ __forceinline__ uint4 rotate_blocks(uint4 cur, uint4 nxt, int s, int lane) {
  const int src = (lane + s) & 31;
  const bool fc = lane + s < 32;
  const unsigned a0 = __shfl_sync(FULL, cur.x, src), b0 = __shfl_sync(FULL, nxt.x, src);
  const unsigned a1 = __shfl_sync(FULL, cur.y, src), b1 = __shfl_sync(FULL, nxt.y, src);
  const unsigned a2 = __shfl_sync(FULL, cur.z, src), b2 = __shfl_sync(FULL, nxt.z, src);
  const unsigned a3 = __shfl_sync(FULL, cur.w, src), b3 = __shfl_sync(FULL, nxt.w, src);
  return make_uint4(fc ? a0 : b0, fc ? a1 : b1, fc ? a2 : b2, fc ? a3 : b3);
}

/* Direction and free path after a p-p event, from the event flight's Philox
   block (createRandomDirectionAllSphere, createRandomFreePath). */
__device__ __forceinline__ void pp_dir(uint4 R, float lam, float& nx, float& ny, float& nz,
                                       float& nf) {
  const float ct = fmaf(u23f(R.x), 2.0f, -1.0f);
  const float st = sqrt_approx(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
  float sp, cp;
  sincos2pi(u23f(R.y), &sp, &cp);
  nx = ct; ny = st * cp; nz = st * sp;
  nf = -lam * __logf(u23f(R.z));
}
/* rotate_blocks for the (free path, direction) a round's lanes drew from
   their blocks: those of this round sit in its rows (flight j at index
   j + 1, RS floats apart), those of the next one in (f2, x2, y2, z2). */
template <int RS>
__device__ __forceinline__ void rotate_dirs(const float* frow, int s, int lane, float f2,
                                            float x2, float y2, float z2, float& f, float& x,
                                            float& y, float& z) {
  const int src = lane + s;
  const int sl = src & 31;
  const float a0 = __shfl_sync(FULL, f2, sl), a1 = __shfl_sync(FULL, x2, sl);
  const float a2 = __shfl_sync(FULL, y2, sl), a3 = __shfl_sync(FULL, z2, sl);
  const bool cur = src < 32;
  const int ri = cur ? src + 1 : 0;
  const float r0 = frow[ri], r1 = frow[RS + ri];
  const float r2 = frow[2 * RS + ri], r3 = frow[3 * RS + ri];
  f = cur ? r0 : a0; x = cur ? r1 : a1; y = cur ? r2 : a2; z = cur ? r3 : a3;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void warp_add_by_task(bool pred, int task, unsigned long long* arr) {
  const unsigned m = __ballot_sync(FULL, pred);
  if (pred) {
    const unsigned peers = __match_any_sync(m, task);
    if ((threadIdx.x & 31) == __ffs(peers) - 1)
      atomicAdd(arr + task, (unsigned long long)__popc(peers));
  }
}

/* Bound of one wait on the staging barrier, in global-timer nanoseconds:
   the copy (at most 96 KB) takes microseconds. */
constexpr unsigned long long kStageWaitNs = 200000000ull;

/* Polls phase 0 of a shared-memory mbarrier until it completes or the global
   timer passes the deadline; returns 1 when it completed. */
__device__ unsigned wait_phase0(unsigned bar_a, unsigned long long deadline) {
  unsigned done = 0;
  for (int it = 0; it < (1 << 26) && !done; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar_a)
        : "memory");
    if (!done && globaltimer() > deadline) break;
  }
  return done;
}

/* Copies the geometry blob into shared memory with one bulk asynchronous
   copy completed on an mbarrier.  The wait is bounded (kStageWaitNs).  On a
   timeout the block sets bit 0 of *err, waits once more, with the same bound,
   for the copy it issued (so that none of its writes can land in shared
   memory after the block has left), and returns false: the block then takes
   no work (the others drain the work queue) and the host returns
   PTG_ERR_TIMEOUT.  issue_copy = false (a test-only option) sets the barrier
   up without issuing the copy, so that the wait runs out with nothing in
   flight. */
__device__ bool stage_blob(const float4* gblob, float4* sblob, int units, int* err,
                           bool issue_copy) {
  __shared__ alignas(8) unsigned long long bar;
  const unsigned bar_a = (unsigned)__cvta_generic_to_shared(&bar);
  const unsigned dst_a = (unsigned)__cvta_generic_to_shared(sblob);
  const unsigned bytes = (unsigned)units * 16u;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes)
                 : "memory");
    if (issue_copy)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              dst_a),
          "l"(gblob), "r"(bytes), "r"(bar_a)
          : "memory");
  }
  const unsigned done = wait_phase0(bar_a, globaltimer() + kStageWaitNs);
  const int ok = __syncthreads_and((int)done);
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      if (issue_copy) wait_phase0(bar_a, globaltimer() + kStageWaitNs);
    }
    __syncthreads();
  }
  return ok != 0;
}

/* Shared-memory accumulators of the adjoint replay: [kAdjBatches][nsurf+1]
   doubles when they fit, else the replay adds to global memory directly. */
constexpr int kAdjSmemDoubles = 2048;

/* rounds of 32 flights one cooperative visit may take before the phonon's
   lane returns to the refill / tally step (a visit also ends where the
   phonon reaches a bath face, is lost or reaches the flight cap) */
constexpr int kCoopRounds = 256;
/* floats between the rows of a warp's cooperative-round block */
constexpr int kRowStride = 36;
/* flights a round tests from its first flight outside the safe ball, in a
   kernel built for BVH grains (every such flight walks the tree and the round
   waits for the slowest walk); the round ends after them */
constexpr int kTestWindow = 4;

/* Kernel phases.  PH_DRAIN pulls (task, particle range) chunks from the
   work queue, one phonon per lane; once the queue is dry a warp holding at
   most coop_lanes live phonons moves them to the tail list (a phonon past
   the list's capacity stays and is finished here).  PH_TAIL runs
   after it: every warp takes one phonon of the tail list at a time into
   lane 0 and advances it with cooperative rounds, so the longest
   trajectories get a warp each instead of sharing one. */
enum { PH_DRAIN = 0, PH_TAIL = 1 };
/* float4 per phonon in the tail list: kTailUnits (kernels.h) */
/* A phonon handed over past this many flights goes to the front of the tail
   list, which the tail phase takes first, the others to the back: a phonon
   that has lasted long is the likeliest to last longer, and the tail ends
   when its longest trajectory does. */
constexpr uint32_t kTailLong = 8192;

/* safe-ball radius searched in a grain with a BVH, in units of the MFP: a
   walk needs about (radius / MFP)^2 flights to leave the ball */
constexpr float kBallCapMfp = 32.0f;

/* Blocks per SM the register budget is cut for: three for the forward and
   listing drain phase (80 registers: a drain 7% shorter on the thin film, 6%
   on the Voronoi polycrystal; the BVH / capped-cylinder variant spills ~70
   bytes and still gains, C4 3833 -> 3677 ms, C3 735 -> 724 ms), two for the
   rest (the tail phase's rounds, and the batched and adjoint kernels, which
   would spill more). */
template <bool SMEM, int MODE, bool BATCH, bool EXT, int PH>
__global__ void __launch_bounds__(kBlock,
                                  (PH == PH_DRAIN && !BATCH && MODE != MODE_ADJOINT) ? 3 : 2)
    k_persistent(GeoF32 gp, RunF32 r) {
  typename std::conditional<BATCH, GeoBatch, Geo<SMEM>>::type G;
  G.lay = gp.lay;
  G.base = gp.blob;
  if (PH == PH_DRAIN && threadIdx.x == 0) atomicMin(r.stats + 5, globaltimer());
  if (SMEM) {
    /* on a timeout the block records the error and takes no work: the host
       reports it */
    if (!stage_blob(gp.blob, sblob, gp.lay.total, r.queue + 1, r.stage_test == 0)) return;
  } else if (EXT && !BATCH && gp.node_stage > 0) {
    /* a blob too large to stage: its BVHs' top levels only */
    if (!stage_blob(gp.blob + gp.lay.bvh_node, sblob, gp.node_stage, r.queue + 1, r.stage_test == 0))
      return;
    G.nstage = gp.node_stage;
  }
  const int lane = threadIdx.x & 31;
  /* geometry and run scalars: kernel-wide, or per lane in a batched launch */
  float X = gp.box[0], Y = gp.box[1], Z = gp.box[2];
  float eps = gp.eps;
  Key2 key = {r.k0, r.k1};
  uint32_t c1 = r.c1;
  int pmask = gp.periodic_mask, nmat = gp.nmaterial;
  float flmax = r.fast_lambda_max;
  /* adjoint replay: per-block accumulators */
  __shared__ double adj_sh[MODE == MODE_ADJOINT ? kAdjSmemDoubles : 1];
  /* cooperative rounds: per warp the rows of the round's 32 free paths and
     directions (fp, dx, dy, dz) and of the start points summed from them
     (x, y, z), 36 floats apart so three lanes reading three rows hit
     different banks */
  __shared__ __align__(16) float coop_rowf[PH == PH_TAIL ? kBlock / 32 : 1][kRowStride * 7];
  float* const crow = coop_rowf[PH == PH_TAIL ? (threadIdx.x >> 5) : 0];
  /* ... and six rows where the lanes' own phonons wait during the rounds */
  __shared__ float4 coop_park[PH == PH_TAIL ? kBlock / 32 : 1][6];
  float4* const park = coop_park[PH == PH_TAIL ? (threadIdx.x >> 5) : 0];
  /* ... and, in kernels built for BVH grains, the warp's local candidate
     list: its entries, its centre and radius, and (count, grain); not in
     the adjoint replay, whose shared accumulators leave no room */
  constexpr bool kUseList = PH == PH_TAIL && EXT && MODE != MODE_ADJOINT;
  constexpr int kLW = kUseList ? kBlock / 32 : 1;
  __shared__ int coop_list[kLW][kList];
  __shared__ float4 coop_lplane[kLW][kList];
  __shared__ float4 coop_ledge[kLW][3 * kList];
  __shared__ float4 coop_lball[kLW];
  __shared__ int4 coop_lmeta[kLW];  /* count, grain, kind (list_bvh) */
  int* const lst = coop_list[kLW > 1 ? (threadIdx.x >> 5) : 0];
  float4* const lpl = coop_lplane[kLW > 1 ? (threadIdx.x >> 5) : 0];
  float4* const led = coop_ledge[kLW > 1 ? (threadIdx.x >> 5) : 0];
  if (kUseList && lane == 0) coop_lmeta[threadIdx.x >> 5] = make_int4(0, -1, 0, 0);
  /* tail phase: phonons the drain left (the counts are final at launch),
     long ones from the front of the list, the others from the back */
  const int nlong = PH == PH_TAIL ? min(r.queue[2], r.tail_cap) : 0;
  const int ntail = PH == PH_TAIL ? nlong + min(r.queue[4], r.tail_cap - nlong) : 0;
  /* accumulators of the sample's geometry: [kAdjBatches][nsurf + 1] at
     adj_off (a batched replay sets both per sample, in global memory) */
  int adj_stride = r.nsurf + 1, adj_off = 0;
  const bool adj_in_smem =
      (MODE == MODE_ADJOINT) && !BATCH && kAdjBatches * (r.nsurf + 1) <= kAdjSmemDoubles;
  if (MODE == MODE_ADJOINT && adj_in_smem) {
    for (int i = threadIdx.x; i < kAdjBatches * (r.nsurf + 1); i += blockDim.x) adj_sh[i] = 0.0;
    __syncthreads();
  }
  float adj_w = 0.0f, adj_len = 0.0f;   /* weight of the sample, path length */
  unsigned adj_npp = 0;                 /* intrinsic events of the sample   */
  int adj_b = 0;                        /* batch of the sample               */
  long long tslot = 0;                  /* trace replay: index of the sample */
  unsigned long long my_mismatch = 0;

  /* warp-uniform chunk cursor */
  int ch_task = -1, ch_next = 0, ch_left = 0;
  bool queue_done = false;
  bool tail_full = false;  /* the tail list refused this warp: stop asking */

  /* lane state */
  bool alive = false;
  float px = 0, py = 0, pz = 0, dx = 1, dy = 0, dz = 0, fp = 0, lam = 0, omr = 0;
  /* safe ball: no surface closer than sqrt(br2) to (bx, by, bz); grain
     ball: no candidate surface of the grain closer than sqrt(gr2) to the
     same centre (box faces excepted), kept until the phonon changes grain */
  float bx = 0, by = 0, bz = 0, br2 = 0, gr2 = 0;
  /* second ball about the same centre: every candidate but the nearest
     (gnear) farther than sqrt(g2r2), so a flight inside it can hit only
     gnear (or a box face) */
  float g2r2 = 0;
  int gnear = -1;
  int grain = 0, last_geom = -1, task = 0;
  uint32_t slo = 0, shi = 0, flight = 0;
  unsigned long long my_flights = 0, my_samples = 0, my_capped = 0, my_lost = 0, my_max = 0;
  unsigned my_full = 0, my_balls = 0;
  unsigned long long my_coop_rounds = 0, my_coop_flights = 0;
  unsigned my_box_tests = 0, my_surf_tests = 0;  /* BVH node boxes, surfaces tested */

  while (true) {
    /* ---- tail phase: lane 0 takes the next phonon of the tail list ----- */
    if (PH == PH_TAIL && !queue_done && !__shfl_sync(FULL, alive, 0)) {
      int c = 0;
      if (lane == 0) c = atomicAdd(r.queue + 3, 1);
      c = __shfl_sync(FULL, c, 0);
      if (c >= ntail) {
        queue_done = true;
      } else if (lane == 0) {
        const int slot =
            r.tail_order ? r.tail_order[c] : (c < nlong ? c : r.tail_cap - 1 - (c - nlong));
        const float4* e = r.tail + (size_t)kTailUnits * slot;
        const float4 e0 = e[0], e1 = e[1], e2 = e[2], e3 = e[3], e4 = e[4];
        px = e0.x; py = e0.y; pz = e0.z; dx = e0.w;
        dy = e1.x; dz = e1.y; fp = e1.z; lam = e1.w;
        bx = e2.x; by = e2.y; bz = e2.z; br2 = e2.w;
        grain = __float_as_int(e3.x); last_geom = __float_as_int(e3.y);
        task = __float_as_int(e3.z); omr = e3.w;
        slo = __float_as_uint(e4.x); shi = __float_as_uint(e4.y);
        flight = __float_as_uint(e4.z); gr2 = e4.w;
        const float4 e6 = e[6];
        g2r2 = e6.x; gnear = __float_as_int(e6.y);
        if (MODE == MODE_ADJOINT) {
          const float4 e5 = e[5];
          adj_w = e5.x; adj_len = e5.y;
          adj_npp = __float_as_uint(e5.z); adj_b = __float_as_int(e5.w);
        }
        alive = true;
      }
    }
    /* ---- refill idle lanes from the warp's chunk ---------------------- */
    unsigned idle = __ballot_sync(FULL, !alive);
    if (PH == PH_DRAIN && !queue_done && idle &&
        (__popc(idle) >= r.regen_threshold || idle == FULL)) {
      while (idle && !queue_done) {
        if (ch_left == 0) {
          int c = 0;
          if (lane == 0) c = atomicAdd(r.queue, 1);
          c = __shfl_sync(FULL, c, 0);
          if (MODE == MODE_ADJOINT || MODE == MODE_TRACE) {
            /* the replay list in chunks of 32 sample ids */
            if ((long long)c * 32 >= r.alist_n) {
              queue_done = true;
              if (lane == 0) atomicMin(r.stats + 6, globaltimer());
              break;
            }
            ch_next = c * 32;
            ch_left = (int)min((long long)32, r.alist_n - (long long)c * 32);
          } else {
            if (c >= r.nchunk) {
              queue_done = true;
              if (lane == 0) atomicMin(r.stats + 6, globaltimer());
              break;
            }
            const int4 q = r.chunk[c];
            ch_task = q.x; ch_next = q.y; ch_left = q.z;
          }
        }
        const int take = min(__popc(idle), ch_left);
        const int rank = __popc(idle & lanemask_lt());
        if (((idle >> lane) & 1u) && rank < take) {
          uint64_t sample;
          const GeoEntry* ge = nullptr;  /* batched launch: the sample's geometry */
          if (MODE == MODE_ADJOINT) {
            const unsigned long long id = r.alist[ch_next + rank];
            if (BATCH) {
              /* batched list entries are (global task << 32) | particle */
              task = (int)(id >> 32);
              ge = r.geos + __ldg(r.task_geo + task);
              sample = (uint64_t)(task - ge->task_base) * (uint64_t)ge->np + (id & 0xffffffffull);
              adj_stride = ge->nsurf + 1;
              adj_off = ge->adj_base;
            } else {
              sample = id;
              task = (int)(sample / (uint64_t)r.np);
            }
            adj_w = r.wsample[task];
            adj_b = (int)(sample % kAdjBatches);
            adj_len = 0.0f;
            adj_npp = 0;
          } else if (MODE == MODE_TRACE) {
            tslot = ch_next + rank;
            sample = r.alist[tslot];
            task = (int)(sample / (uint64_t)r.np);
          } else if (BATCH) {
            const int64_t p = (int64_t)r.rank + (int64_t)(ch_next + rank) * r.nranks;
            task = ch_task;
            ge = r.geos + __ldg(r.task_geo + task);
            sample = (uint64_t)(task - ge->task_base) * (uint64_t)ge->np + (uint64_t)p;
          } else {
            const int64_t p = (int64_t)r.rank + (int64_t)(ch_next + rank) * r.nranks;
            sample = (uint64_t)ch_task * (uint64_t)r.np + (uint64_t)p;
            task = ch_task;
          }
          if (BATCH && ge) {
            G.base = ge->blob;
            G.lay = ge->lay;
            X = ge->box[0]; Y = ge->box[1]; Z = ge->box[2];
            eps = ge->eps;
            key.k0 = ge->k0; key.k1 = ge->k1;
            c1 = ge->c1;
            pmask = ge->periodic_mask;
            nmat = ge->nmaterial;
            flmax = ge->fast_lambda_max;
          }
          slo = (uint32_t)sample;
          shi = (uint32_t)(sample >> 32);
          const float4 T = r.task[task];
          lam = T.x;
          omr = T.w;
          /* emission: createRandomPosition / createRandomDirectionPhi,
             src/RTMCphon.f90:1845-1871; flight 0 draws y, z, phi, free path */
          const uint4 R0 = philox10(0u, c1, slo, shi, key);
          float sc0 = gp.scope[0], sc1 = gp.scope[1];
          int kgrain = gp.kind_grain, gfill = gp.igrain_fill;
          if (BATCH) {
            const GeoEntry* e = r.geos + __ldg(r.task_geo + task);
            sc0 = e->scope[0]; sc1 = e->scope[1];
            kgrain = e->kind_grain; gfill = e->igrain_fill;
          }
          px = 0.0f;
          py = u23f(R0.x) * Y * sc0;
          pz = u23f(R0.y) * Z * sc1;
          float sp, cp;
          sincos2pi(u23f(R0.z), &sp, &cp);
          dx = T.y;
          dy = T.z * cp;
          dz = T.z * sp;
          fp = isinf(lam) ? lam : -lam * __logf(u23f(R0.w));
          /* start grain: nearest incident generatrix (voronoi,
             src/RTMCphon.f90:2100-2118) or the last incident polygon
             containing the point, else the fill grain (bricks, :2131-2163) */
          grain = 0;
          if (kgrain == 1) {
            float dmin = 3.0e38f;
            for (int i = 0; i < G.lay.nstart; ++i) {
              const float4 s = G.start(i);
              const float a = px - s.x, b = py - s.y, c = pz - s.z;
              const float d2 = fmaf(a, a, fmaf(b, b, c * c));
              if (d2 < dmin) { dmin = d2; grain = __float_as_int(s.w); }
            }
          } else {
            grain = gfill;
            for (int i = 0; i < G.lay.nstart; ++i) {
              const float4 s = G.start(i);
              const int sid = __float_as_int(s.x);
              const int4 B = G.hotB(sid);
              if (inside_edges(G, B.y, B.z, px, py, pz, 0.0f)) grain = __float_as_int(s.y);
            }
          }
          last_geom = -1;
          br2 = 0.0f;
          gr2 = 0.0f;
          g2r2 = 0.0f;
          gnear = -1;
          flight = 0;
          alive = true;
          my_samples += 1;
          if (MODE == MODE_TRACE) trace_put(r, tslot, 0u, px, py, pz);
        }
        ch_next += take;
        ch_left -= take;
        idle = __ballot_sync(FULL, !alive);
      }
    }
    if (!__any_sync(FULL, alive)) {
      if (queue_done) break;
      continue;
    }
    /* ---- drain phase, queue dry: live phonons go to the tail list (the
       diffusive ones and, as well, the few long-MFP ones, which would
       otherwise hold their warp, and the drain launch, to the end) */
    if (PH == PH_DRAIN && !BATCH && MODE != MODE_TRACE && queue_done && r.coop_lanes > 0 &&
        !tail_full && __popc(__ballot_sync(FULL, alive)) <= r.coop_lanes) {
      const unsigned mw = __ballot_sync(FULL, alive);
      if (mw) {
        /* a slot is reserved from one counter of all requests (queue[5])
           before the phonon picks its end of the list: the phonons admitted
           number at most tail_cap, so the long ones, filling the list from
           the front, and the others, filling it from the back, never meet
           whatever the list's size; a phonon past the capacity stays here */
        const int fw = __ffs(mw) - 1;
        int bw = 0;
        if (lane == fw) bw = atomicAdd(r.queue + 5, __popc(mw));
        bw = __shfl_sync(FULL, bw, fw);
        const unsigned mv =
            mw & __ballot_sync(FULL, bw + __popc(mw & lanemask_lt()) < r.tail_cap);
        if (mv != mw) tail_full = true;
        const unsigned ml = mv & __ballot_sync(FULL, flight >= kTailLong);
        const unsigned ms = mv & ~ml;
        const int fl = ml ? __ffs(ml) - 1 : 0, fs = ms ? __ffs(ms) - 1 : 0;
        int bl = 0, bs = 0;
        if (ml && lane == fl) bl = atomicAdd(r.queue + 2, __popc(ml));
        if (ms && lane == fs) bs = atomicAdd(r.queue + 4, __popc(ms));
        bl = __shfl_sync(FULL, bl, fl);
        bs = __shfl_sync(FULL, bs, fs);
        const bool lng = (ml >> lane) & 1u;
        const int idx = lng ? bl + __popc(ml & lanemask_lt()) : bs + __popc(ms & lanemask_lt());
        const int slot = lng ? idx : r.tail_cap - 1 - idx;
        /* past the list's capacity a phonon stays here */
        if (((mv >> lane) & 1u) && idx < r.tail_cap && slot >= 0 && slot < r.tail_cap) {
          float4* e = r.tail + (size_t)kTailUnits * slot;
          e[0] = make_float4(px, py, pz, dx);
          e[1] = make_float4(dy, dz, fp, lam);
          e[2] = make_float4(bx, by, bz, br2);
          e[3] = make_float4(__int_as_float(grain), __int_as_float(last_geom),
                             __int_as_float(task), omr);
          e[4] = make_float4(__uint_as_float(slo), __uint_as_float(shi), __uint_as_float(flight),
                             gr2);
          e[6] = make_float4(g2r2, __int_as_float(gnear), 0.0f, 0.0f);
          if (MODE == MODE_ADJOINT)
            e[5] = make_float4(adj_w, adj_len, __uint_as_float(adj_npp), __int_as_float(adj_b));
          atomicAdd(r.stats + 16, (unsigned long long)flight);
          alive = false;
        }
        if (!__any_sync(FULL, alive)) {
          if (queue_done) break;
          continue;
        }
      }
    }

    int end_side = -1;  /* -1 still running, 0 lost, 1 x-, 2 x+ */

    /* ---- tail phase: warp-cooperative flights for lane 0's phonon -------
       The warp's 32 lanes advance the phonon 32 flights per round: lane j
       draws the Philox block of flight f+1+j, the start point of every
       flight is the serial sum of the earlier flights (in their order, with
       the rounding of the one-lane path), and each lane runs the full
       intersection test of its own flight unless the flight stays in the
       safe ball.  The first flight that hits a surface, leaves the box or
       reaches the cap ends the round; the flights before it are p-p events.
       A surface or side-face event is taken by the whole warp
       (surface_hit) and the rounds go on from it; at a bath face (and in
       the adjoint replay at any surface) the hit flight's Philox block and
       nearest surface are handed to the phonon's lane, which processes the
       event below. */
    bool coop = false;       /* this lane was advanced cooperatively          */
    bool pre = false;        /* ... up to a surface hit: preR / pre_tb / pre_sb */
    bool skip_full = false;  /* ... up to the round limit: no event this pass  */
    uint4 preR = make_uint4(0u, 0u, 0u, 0u);
    float pre_tb = 0.0f;
    int pre_sb = -1;
    if (PH == PH_TAIL) {
      const unsigned todo0 = __ballot_sync(FULL, lane == 0 && alive);
      const int max_rounds = kCoopRounds;
      if (todo0) {
        /* the warp's phonon (in the tail phase lane 0 holds the only one)
           waits in the warp's park row while the warp runs the rounds, so
           its registers serve the rounds; every lane reads it (broadcast
           loads) and lane 0 writes it back */
        if (lane == 0) {
          park[0] = make_float4(px, py, pz, dx);
          park[1] = make_float4(dy, dz, fp, lam);
          park[2] = make_float4(bx, by, bz, br2);
          park[3] = make_float4(__int_as_float(grain), __int_as_float(last_geom),
                                __int_as_float(task), omr);
          park[4] = make_float4(__uint_as_float(slo), __uint_as_float(shi),
                                __uint_as_float(flight), gr2);
          park[5] = make_float4(g2r2, __int_as_float(gnear), 0.0f, 0.0f);
        }
        __syncwarp();
        unsigned todo = todo0;
        while (todo) {
          const int L = __ffs(todo) - 1;
          todo &= todo - 1;
          const float4 s0 = park[0], s1 = park[1], s2 = park[2], s3 = park[3];
          const float4 s4 = park[4];
          const float4 s5 = park[5];
          float cpx = s0.x, cpy = s0.y, cpz = s0.z;
          float cdx = s0.w, cdy = s1.x, cdz = s1.y, cfp = s1.z;
          const float clam = s1.w;
          uint32_t cfl = __float_as_uint(s4.z);
          const uint32_t cslo = __float_as_uint(s4.x), cshi = __float_as_uint(s4.y);
          int cgrain = __float_as_int(s3.x);
          int clast = __float_as_int(s3.y);
          /* the phonon's safe ball: flights ending inside it skip the test */
          float cbx = s2.x, cby = s2.y, cbz = s2.z, cbr2 = s2.w, cgr2 = s4.w;
          float cg2r2 = s5.x;
          int cnear = __float_as_int(s5.y);
          float clen = 0.0f;
          unsigned cnpp = 0, ctaken = 0, crounds = 0;
          int stop = 0;  /* 0 round limit, 1 surface hit, 2 lost or capped */
          uint4 sR = make_uint4(0u, 0u, 0u, 0u);
          float stb = 0.0f;
          int ssb = -1;
          /* the blocks of the next round are drawn while this one runs,
             assuming it advances all 32 flights (counters alone fix them);
             a round that advances fewer passes the ones it has on
             (rotate_blocks) */
          uint4 Rnext = philox10(cfl + 1u + (uint32_t)lane, c1, cslo, cshi, key);
          /* ... and so are the directions and free paths they give, which
             the round writes to its rows without waiting for them */
          float nx, ny, nz, nf;
          pp_dir(Rnext, clam, nx, ny, nz, nf);
          for (int round = 0; round < max_rounds; ++round) {
            ++crounds;
            const uint4 R = Rnext;
            Rnext = philox10(cfl + 33u + (uint32_t)lane, c1, cslo, cshi, key);
            float nx2, ny2, nz2, nf2;
            pp_dir(Rnext, clam, nx2, ny2, nz2, nf2);
            /* flight `lane` starts with the state the previous flight drew:
               the rows hold the (free path, direction) of the round's 32
               flights.  The start point of flight j is the chain p,
               fma(fp_0, d_0, p), ... after j steps, the same for every lane,
               so lane c < 3 runs coordinate c's chain alone (two 4-wide
               loads, four fmas and one 4-wide store of the chain per four
               flights) and every lane then reads its own start point */
            float* const frow = crow;
            /* (lane 31's entry, index 32, serves rotate_dirs) */
            frow[lane + 1] = nf;
            frow[kRowStride + lane + 1] = nx;
            frow[2 * kRowStride + lane + 1] = ny;
            frow[3 * kRowStride + lane + 1] = nz;
            if (lane == 0) {
              frow[0] = cfp;
              frow[kRowStride] = cdx;
              frow[2 * kRowStride] = cdy;
              frow[3 * kRowStride] = cdz;
            }
            __syncwarp();
            const float sfp = frow[lane], sdx = frow[kRowStride + lane];
            const float sdy = frow[2 * kRowStride + lane], sdz = frow[3 * kRowStride + lane];
            {
              const int cc = lane < 3 ? lane : 2;
              const float* const drow = frow + kRowStride * (cc + 1);
              float* const qrow = frow + kRowStride * (cc + 4);
              float a = cc == 0 ? cpx : (cc == 1 ? cpy : cpz);
              /* the rows' loads run two blocks ahead of the chain: a block's
                 loads are issued before the previous block's store, which
                 the compiler may not move them across */
              float4 fa = *reinterpret_cast<const float4*>(frow);
              float4 da = *reinterpret_cast<const float4*>(drow);
              float4 fb = *reinterpret_cast<const float4*>(frow + 4);
              float4 db = *reinterpret_cast<const float4*>(drow + 4);
#pragma unroll
              for (int b = 0; b < 32; b += 4) {
                const float4 f = fa, d = da;
                fa = fb;
                da = db;
                if (b + 8 < 32) {
                  fb = *reinterpret_cast<const float4*>(frow + b + 8);
                  db = *reinterpret_cast<const float4*>(drow + b + 8);
                }
                float4 q;
                a = fmaf(f.x, d.x, a);
                q.x = a;
                a = fmaf(f.y, d.y, a);
                q.y = a;
                a = fmaf(f.z, d.z, a);
                q.z = a;
                a = fmaf(f.w, d.w, a);
                q.w = a;
                if (lane < 3) *reinterpret_cast<float4*>(qrow + b) = q;
              }
            }
            __syncwarp();
            const int jq = lane > 0 ? lane - 1 : 0;
            const float qx = lane == 0 ? cpx : frow[4 * kRowStride + jq];
            const float qy = lane == 0 ? cpy : frow[5 * kRowStride + jq];
            const float qz = lane == 0 ? cpz : frow[6 * kRowStride + jq];
            __syncwarp();  /* the next round rewrites the rows */
            const bool inbox = qx >= -eps && qx <= X + eps && qy >= -eps && qy <= Y + eps &&
                               qz >= -eps && qz <= Z + eps;
            const bool capd = (unsigned long long)cfl + (unsigned)lane >= r.max_flights;
            /* a flight that starts and ends in the safe ball stays in it (the
               ball is convex and holds no surface) and ends in a p-p event;
               the others take the intersection test */
            const float ex = fmaf(sfp, sdx, qx) - cbx, ey = fmaf(sfp, sdy, qy) - cby;
            const float ez = fmaf(sfp, sdz, qz) - cbz;
            const float sx = qx - cbx, sy = qy - cby, sz = qz - cbz;
            const float de2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            const float ds2 = fmaf(sx, sx, fmaf(sy, sy, sz * sz));
            const bool in_ball = de2 < cbr2 && ds2 < cbr2;
            /* in the grain ball only the box faces can be hit, in the second
               ball only they and the grain's nearest candidate */
            const bool in_gball = de2 < cgr2 && ds2 < cgr2;
            const bool in_g2 = de2 < cg2r2 && ds2 < cg2r2;
            /* ... and within the local list's radius only the listed ones */
            bool in_list = false;
            int lkind = 0;
            int ln = 0;
            if (kUseList) {
              const int4 lm = coop_lmeta[threadIdx.x >> 5];
              const float4 lc = coop_lball[threadIdx.x >> 5];
              const float ru = lc.w - 4.0f * eps;
              lkind = lm.z;
              const float lx = fmaf(sfp, sdx, qx) - lc.x, ly = fmaf(sfp, sdy, qy) - lc.y;
              const float lz = fmaf(sfp, sdz, qz) - lc.z;
              const float mx = qx - lc.x, my = qy - lc.y, mz = qz - lc.z;
              ln = lm.x;
              in_list = lm.y == cgrain && ru > 0.0f &&
                        fmaf(lx, lx, fmaf(ly, ly, lz * lz)) < ru * ru &&
                        fmaf(mx, mx, fmaf(my, my, mz * mz)) < ru * ru;
            }
            /* in kernels built for BVH grains a round tests at most
               kTestWindow flights from its first one that needs the whole
               grain's search */
            const unsigned needm = __ballot_sync(FULL, !in_ball && !in_gball && !in_g2 && !in_list);
            const int jw = (EXT && needm) ? min(32, __ffs(needm) - 1 + kTestWindow) : 32;
            float tb = 3.0e38f;
            int sb = -1;
            if (!in_ball && lane < jw) {
              slab_exit(qx, qy, qz, sdx, sdy, sdz, X, Y, Z, tb, sb);
              if (cgrain > 0 && !in_gball) {
                if (in_g2)
                  test_near<EXT>(G, cnear, qx, qy, qz, sdx, sdy, sdz, lane == 0 ? clast : -1, eps, Z,
                                 tb, sb, my_surf_tests);
                else if (kUseList && in_list)
                  scan_list<EXT>(G, lst, lpl, led, ln, lkind, qx, qy, qz, sdx, sdy, sdz,
                                 lane == 0 ? clast : -1, eps, Z, sfp, tb, sb, my_surf_tests);
                else
                  scan_grain<EXT>(G, cgrain, qx, qy, qz, sdx, sdy, sdz, lane == 0 ? clast : -1, eps,
                                  Z, sfp, tb, sb, my_box_tests, my_surf_tests);
              }
            }
            const bool brk = !inbox || capd;
            const unsigned sm =
                __ballot_sync(FULL, lane < jw && (brk || (!in_ball && !(sfp < tb))));
            const int j = sm ? __ffs(sm) - 1 : jw;
            if (MODE == MODE_ADJOINT) {
              float l = lane < j ? sfp : 0.0f;
              for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(FULL, l, o);
              clen += l;
              cnpp += (unsigned)j;
            }
            ctaken += (unsigned)j;
            if (sm) {
              cpx = __shfl_sync(FULL, qx, j); cpy = __shfl_sync(FULL, qy, j);
              cpz = __shfl_sync(FULL, qz, j);
              cdx = __shfl_sync(FULL, sdx, j); cdy = __shfl_sync(FULL, sdy, j);
              cdz = __shfl_sync(FULL, sdz, j); cfp = __shfl_sync(FULL, sfp, j);
              cfl += (uint32_t)j;
              if (j > 0) clast = -1;
              stop = __shfl_sync(FULL, brk ? 2 : 1, j);
              if (stop == 1) {
                sR.x = __shfl_sync(FULL, R.x, j); sR.y = __shfl_sync(FULL, R.y, j);
                sR.z = __shfl_sync(FULL, R.z, j); sR.w = __shfl_sync(FULL, R.w, j);
                stb = __shfl_sync(FULL, tb, j);
                ssb = __shfl_sync(FULL, sb, j);
                if (MODE != MODE_ADJOINT && ssb > 1) {
                  /* a surface or a side face, not a bath: every lane takes
                     the event (the same inputs, the same result) and the
                     rounds go on from it; a bath face ends the visit */
                  ++cfl;
                  ++ctaken;
                  const AdjAcc none{nullptr, nullptr, 0.0f, 0, false};
                  surface_hit<MODE, EXT>(G, stb, ssb, u23f(sR.x), u23f(sR.y), u23f(sR.z),
                                         u23f(sR.w), Y, Z, pmask, nmat, s3.w, clam, cfl, c1, cslo,
                                         cshi, key, none, cpx, cpy, cpz, cdx, cdy, cdz, cfp, cgrain,
                                         cgr2, cg2r2, clast);
                  cbr2 = 0.0f;
                  stop = 0;
                  Rnext = rotate_blocks(R, Rnext, j + 1, lane);
                  rotate_dirs<kRowStride>(frow, j + 1, lane, nf2, nx2, ny2, nz2, nf, nx, ny, nz);
                  continue;
                }
              }
              break;
            }
            if (j < 32) {
              /* the window's flights all end in p-p events: the state at the
                 start of flight j */
              cpx = __shfl_sync(FULL, qx, j); cpy = __shfl_sync(FULL, qy, j);
              cpz = __shfl_sync(FULL, qz, j);
              cdx = __shfl_sync(FULL, sdx, j); cdy = __shfl_sync(FULL, sdy, j);
              cdz = __shfl_sync(FULL, sdz, j); cfp = __shfl_sync(FULL, sfp, j);
            } else {
              /* all 32 flights end in p-p events: the state after the last */
              cpx = __shfl_sync(FULL, fmaf(sfp, sdx, qx), 31);
              cpy = __shfl_sync(FULL, fmaf(sfp, sdy, qy), 31);
              cpz = __shfl_sync(FULL, fmaf(sfp, sdz, qz), 31);
              cdx = __shfl_sync(FULL, nx, 31); cdy = __shfl_sync(FULL, ny, 31);
              cdz = __shfl_sync(FULL, nz, 31); cfp = __shfl_sync(FULL, nf, 31);
            }
            cfl += (uint32_t)j;
            if (j != 32) {
              Rnext = rotate_blocks(R, Rnext, j, lane);
              rotate_dirs<kRowStride>(frow, j, lane, nf2, nx2, ny2, nz2, nf, nx, ny, nz);
            } else {
              nf = nf2; nx = nx2; ny = ny2; nz = nz2;
            }
            /* a new ball where the walk left the grain ball: while it stays
               in the grain ball only the box faces can be hit, and a slab
               test per flight costs less than renewing the safe ball each
               time the walk leaves it (the old safe ball stays valid) */
            if (!__shfl_sync(FULL, in_gball, j - 1) && r.fast_steps > 0) {
              float dg, dg2, d;
              if (kUseList && cgrain > 0 && G.bvh_root(cgrain) >= 0) {
                /* from the local list, built anew (one tree search) in
                   another grain or where the list's edge bounds the ball */
                const int4 lm = coop_lmeta[threadIdx.x >> 5];
                const float4 lc = coop_lball[threadIdx.x >> 5];
                bool fresh = lm.y != cgrain;
                if (!fresh) {
                  d = safety_list<EXT>(G, lst, lm.x, lc, cpx, cpy, cpz, X, Y, Z, eps, lane, dg, dg2,
                                       cnear);
                  /* a ball bounded by the list's edge, not by a listed
                     surface, and short of half the search radius: a new
                     list about this point */
                  const float wx = cpx - lc.x, wy = cpy - lc.y, wz = cpz - lc.z;
                  const float du = lc.w - sqrt_approx(fmaf(wx, wx, fmaf(wy, wy, wz * wz)));
                  fresh = cnear < 0 && du < 0.5f * kListMfp * clam;
                }
                if (fresh) {
                  /* the search radius: kListMfp MFPs, or a quarter more than
                     the last list's if that one filled up in this grain
                     (fewer replacements in a dense grain) */
                  const float rt = kListMfp * clam;
                  const float r0 = (lm.y == cgrain && lm.x == kList) ? fminf(rt, 1.25f * lc.w) : rt;
                  int n, ap;
                  const float R = list_bvh<EXT>(G, G.bvh_root(cgrain), cpx, cpy, cpz, r0, lane, lst,
                                                lpl, led, n, ap);
                  const float4 nc = make_float4(cpx, cpy, cpz, R);
                  if (lane == 0) {
                    coop_lball[threadIdx.x >> 5] = nc;
                    coop_lmeta[threadIdx.x >> 5] = make_int4(n, cgrain, ap, 0);
                  }
                  __syncwarp();
                  d = safety_list<EXT>(G, lst, n, nc, cpx, cpy, cpz, X, Y, Z, eps, lane, dg, dg2,
                                       cnear);
                }
              } else {
                d = safety<EXT>(G, cgrain, cpx, cpy, cpz, X, Y, Z, eps, kBallCapMfp * clam, dg, dg2,
                                cnear);
              }
              cbx = cpx; cby = cpy; cbz = cpz;
              cbr2 = d > 0.0f ? d * d : 0.0f;
              cgr2 = dg > 0.0f ? dg * dg : 0.0f;
              cg2r2 = (dg2 > 0.0f && cnear >= 0) ? dg2 * dg2 : 0.0f;
            }
            clast = -1;
          }
          if (lane == L) {
            park[0] = make_float4(cpx, cpy, cpz, cdx);
            park[1] = make_float4(cdy, cdz, cfp, clam);
            park[2] = make_float4(cbx, cby, cbz, cbr2);
            park[3] = make_float4(__int_as_float(cgrain), __int_as_float(clast),
                                        s3.z, s3.w);
            park[4] = make_float4(s4.x, s4.y, __uint_as_float(cfl), cgr2);
            park[5] = make_float4(cg2r2, __int_as_float(cnear), 0.0f, 0.0f);
            if (MODE == MODE_ADJOINT) {
              adj_len += clen;
              adj_npp += cnpp;
            }
            coop = true;
            if (stop == 1) {
              pre = true;
              preR = sR;
              pre_tb = stb;
              pre_sb = ssb;
            } else if (stop == 0) {
              skip_full = true;
            }
            my_coop_rounds += crounds;
            my_coop_flights += ctaken;
          }
        }
        /* lane 0 takes its phonon back (it wrote the row last); the other
           lanes, which hold no phonon, read the same row, so that no state
           of theirs has to live through the rounds */
        __syncwarp();
        const float4 s0 = park[0], s1 = park[1], s2 = park[2];
        const float4 s3 = park[3], s4 = park[4], s5 = park[5];
        px = s0.x; py = s0.y; pz = s0.z; dx = s0.w;
        dy = s1.x; dz = s1.y; fp = s1.z; lam = s1.w;
        bx = s2.x; by = s2.y; bz = s2.z; br2 = s2.w;
        grain = __float_as_int(s3.x); last_geom = __float_as_int(s3.y);
        task = __float_as_int(s3.z); omr = s3.w;
        slo = __float_as_uint(s4.x); shi = __float_as_uint(s4.y); flight = __float_as_uint(s4.z);
        gr2 = s4.w;
        g2r2 = s5.x; gnear = __float_as_int(s5.y);
      }
    }

    bool paused = false;  /* stopped by the step limit while still in its ball */
    {
      /* ---- safe-ball p-p flights: the segment to the next p-p point stays
         inside the safe ball (convex), so no surface is crossed.  Four
         flights at a time: their Philox blocks, new directions and free
         paths do not depend on the phonon state and are computed together;
         only the position / ball test chain is serial.  Every lane takes
         part in the loop control (the ballots): past fast_steps flights the
         warp goes on only while at least half of its live lanes are still in
         their balls, and never past 4 x fast_steps, so a few lanes deep in
         large balls do not hold the others' full flights back. ---- */
      bool fast_more = alive && MODE != MODE_TRACE && br2 > 0.0f && !coop;
      const int nalive = __popc(__ballot_sync(FULL, alive));
      for (int g = 0;; g += 4) {
        const bool go = fast_more && flight + 4u <= r.max_flights;
        const unsigned gm = __ballot_sync(FULL, go);
        if (!gm) break;
        if (g >= r.fast_steps && (g >= 4 * r.fast_steps || 2 * __popc(gm) < nalive)) {
          paused = go;
          break;
        }
        if (!go) continue;
        uint4 B[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) B[j] = philox10(flight + 1u + j, c1, slo, shi, key);
        float nx[4], ny[4], nz[4], nf[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float ct = fmaf(u23f(B[j].x), 2.0f, -1.0f);
          const float st = sqrt_approx(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
          float sp, cp;
          sincos2pi(u23f(B[j].y), &sp, &cp);
          nx[j] = ct;
          ny[j] = st * cp;
          nz[j] = st * sp;
          nf[j] = -lam * __logf(u23f(B[j].z));
        }
        /* the position advances with the same rounding as a full flight's
           p-p event, so the trajectory does not depend on which path took
           a flight */
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          /* predicated: no branch per step */
          const float qx = fmaf(fp, dx, px), qy = fmaf(fp, dy, py), qz = fmaf(fp, dz, pz);
          const float ex = qx - bx, ey = qy - by, ez = qz - bz;
          const bool acc = fast_more && (fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < br2);
          if (MODE == MODE_ADJOINT) {
            adj_len += acc ? fp : 0.0f;
            adj_npp += acc ? 1u : 0u;
          }
          flight += acc ? 1u : 0u;
          px = acc ? qx : px; py = acc ? qy : py; pz = acc ? qz : pz;
          dx = acc ? nx[j] : dx; dy = acc ? ny[j] : dy; dz = acc ? nz[j] : dz;
          fp = acc ? nf[j] : fp;
          fast_more = acc;
        }
      }
    }
    if (alive) {
      /* a lane paused in its ball waits for the next iteration; any other
         lane takes one flight with the full test now */
      if (!paused && !skip_full) {
        /* ---- one free flight with the intersection test (already run by
           the cooperative round when it handed over a hit) -------------- */
        bool go = false;
        uint4 R = preR;
        float tb = pre_tb;
        int sb = pre_sb;
        if (pre) {
          ++flight;
          go = true;
        } else if (!(px >= -eps && px <= X + eps && py >= -eps && py <= Y + eps &&
                     pz >= -eps && pz <= Z + eps)) {
          end_side = 0;
        } else if (flight >= r.max_flights) {
          end_side = 0;
          my_capped += 1;
        } else {
          ++flight;
          ++my_full;
          R = philox10(flight, c1, slo, shi, key);
          slab_exit(px, py, pz, dx, dy, dz, X, Y, Z, tb, sb);
          const float ex = fmaf(fp, dx, px) - bx, ey = fmaf(fp, dy, py) - by;
          const float ez = fmaf(fp, dz, pz) - bz;
          const float sx = px - bx, sy = py - by, sz = pz - bz;
          const float fe2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
          const float fs2 = fmaf(sx, sx, fmaf(sy, sy, sz * sz));
          const bool in_gball = fe2 < gr2 && fs2 < gr2;
          /* the second ball pays here where the grains' scans walk BVHs or
             test capped cylinders; in a grain of a few plain surfaces its
             extra branch costs more than it saves */
          if (grain > 0 && !in_gball) {
            if (EXT && fe2 < g2r2 && fs2 < g2r2)
              test_near<EXT>(G, gnear, px, py, pz, dx, dy, dz, last_geom, eps, Z, tb, sb,
                             my_surf_tests);
            else
              scan_grain<EXT>(G, grain, px, py, pz, dx, dy, dz, last_geom, eps, Z, fp, tb, sb,
                              my_box_tests, my_surf_tests);
          }
          go = true;
        }
        if (go) {
          const float u0 = u23f(R.x), u1 = u23f(R.y), u2 = u23f(R.z), u3 = u23f(R.w);
          if (fp < tb) {
            /* intrinsic scattering: isotropic direction, new free path */
            if (MODE == MODE_ADJOINT) {
              adj_len += fp;
              adj_npp += 1u;
            }
            px = fmaf(fp, dx, px);
            py = fmaf(fp, dy, py);
            pz = fmaf(fp, dz, pz);
            const float ct = fmaf(u0, 2.0f, -1.0f);
            const float st = sqrt_approx(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
            float sp, cp;
            sincos2pi(u1, &sp, &cp);
            dx = ct;
            dy = st * cp;
            dz = st * sp;
            fp = -lam * __logf(u2);
            last_geom = -1;
            br2 = 0.0f;
            if (MODE != MODE_TRACE && r.fast_steps > 0 && lam < flmax) {
              float dg, dg2;
              int nr;
              const float d =
                  safety<EXT>(G, grain, px, py, pz, X, Y, Z, eps, kBallCapMfp * lam, dg, dg2, nr);
              ++my_balls;
              if (dg > 0.0f) {
                bx = px; by = py; bz = pz;
                br2 = d > 0.0f ? d * d : 0.0f;
                gr2 = dg * dg;
                g2r2 = (dg2 > 0.0f && nr >= 0) ? dg2 * dg2 : 0.0f;
                gnear = nr;
              }
            }
          } else {
            if (MODE == MODE_ADJOINT) adj_len += tb;
            const AdjAcc acc{adj_sh, r.adj, adj_w, adj_off + adj_b * adj_stride, adj_in_smem};
            end_side = surface_hit<MODE, EXT>(G, tb, sb, u0, u1, u2, u3, Y, Z, pmask, nmat, omr, lam,
                                              flight, c1, slo, shi, key, acc, px, py, pz, dx, dy, dz,
                                              fp, grain, gr2, g2r2, last_geom);
            br2 = 0.0f;
          }
          if (MODE == MODE_TRACE) trace_put(r, tslot, flight, px, py, pz);
        }
      }
    }
#ifdef PT_CHECK
    if (alive && !(isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(dx) && isfinite(dy) &&
                   isfinite(dz) && !isnan(fp)))
      check_fail(2, task);
#endif
    /* ---- tallies ------------------------------------------------------- */
    const bool fin = alive && end_side >= 0;
    const bool trans = fin && (end_side == 2 || (end_side == 0 && r.ref_quirks));
    const bool lostp = fin && end_side == 0;
    if (MODE != MODE_ADJOINT) {
      warp_add_by_task(trans, task, r.counts);
      warp_add_by_task(lostp, task, r.lost);
    }
    if (MODE == MODE_LIST) {
      /* compact the ids of transmitted phonons (exit through x+) */
      const bool put = fin && end_side == 2;
      const unsigned m = __ballot_sync(FULL, put);
      if (m) {
        unsigned long long base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(r.stats + 10, (unsigned long long)__popc(m));
        base = __shfl_sync(FULL, base, __ffs(m) - 1);
        const unsigned long long at = base + __popc(m & lanemask_lt());
        if (put && at < r.tlist_cap) {
          unsigned long long id = ((unsigned long long)shi << 32) | slo;
          if (BATCH) {
            /* (global task << 32) | particle: the replay finds the geometry */
            const GeoEntry* e = r.geos + __ldg(r.task_geo + task);
            id = ((unsigned long long)task << 32) |
                 (id - (unsigned long long)(task - e->task_base) * (unsigned long long)e->np);
          }
          r.tlist[at] = id;
        }
      }
    }
    if (MODE == MODE_TRACE && fin) {
      r.trace_npos[tslot] = (long long)flight + 1;
      r.trace_end[tslot] = end_side;
    }
    if (MODE == MODE_ADJOINT && fin) {
      if (end_side == 2) {
        /* d log P / d s of the exponential free paths at rate s / lambda */
        const double v = (double)adj_w * ((double)adj_npp - (double)adj_len / (double)lam);
        const int idx = adj_off + adj_b * adj_stride + adj_stride - 1;
        if (!isinf(lam)) {
          if (adj_in_smem) atomicAdd(&adj_sh[idx], v);
          else atomicAdd(&r.adj[idx], v);
        }
      } else {
        my_mismatch += 1;
      }
    }
    if (fin) {
      my_flights += flight;
      my_lost += lostp ? 1 : 0;
      my_max = max(my_max, (unsigned long long)flight);
      alive = false;
    }
  }
  /* warp totals */
  unsigned long long v0 = my_flights, v1 = my_lost, v2 = my_capped, v3 = my_samples, v4 = my_max;
  unsigned long long v5 = my_full, v6 = my_balls, v7 = my_coop_rounds, v8 = my_coop_flights;
  unsigned long long v9 = my_box_tests, v10 = my_surf_tests;
  for (int o = 16; o > 0; o >>= 1) {
    v5 += __shfl_xor_sync(FULL, v5, o);
    v6 += __shfl_xor_sync(FULL, v6, o);
    v7 += __shfl_xor_sync(FULL, v7, o);
    v8 += __shfl_xor_sync(FULL, v8, o);
    v9 += __shfl_xor_sync(FULL, v9, o);
    v10 += __shfl_xor_sync(FULL, v10, o);
    v0 += __shfl_xor_sync(FULL, v0, o);
    v1 += __shfl_xor_sync(FULL, v1, o);
    v2 += __shfl_xor_sync(FULL, v2, o);
    v3 += __shfl_xor_sync(FULL, v3, o);
    v4 = max(v4, __shfl_xor_sync(FULL, v4, o));
  }
  if (MODE == MODE_ADJOINT) {
    for (int o = 16; o > 0; o >>= 1) my_mismatch += __shfl_xor_sync(FULL, my_mismatch, o);
    if (lane == 0 && my_mismatch) atomicAdd(r.stats + 11, my_mismatch);
  }
  if (lane == 0) {
    if (v0) atomicAdd(r.stats + 0, v0);
    if (PH == PH_TAIL && v0) atomicAdd(r.stats + 17, v0);
    if (v1) atomicAdd(r.stats + 1, v1);
    if (v2) atomicAdd(r.stats + 2, v2);
    if (v3) atomicAdd(r.stats + 3, v3);
    atomicMax(r.stats + 4, v4);
    atomicMax(r.stats + 7, globaltimer());
    if (v5) atomicAdd(r.stats + 8, v5);
    if (v6) atomicAdd(r.stats + 9, v6);
    if (v7) atomicAdd(r.stats + 12, v7);
    if (v8) atomicAdd(r.stats + 13, v8);
    if (v9) atomicAdd(r.stats + 14, v9);
    if (v10) atomicAdd(r.stats + 15, v10);
  }
  if (MODE == MODE_ADJOINT && adj_in_smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < kAdjBatches * (r.nsurf + 1); i += blockDim.x)
      if (adj_sh[i] != 0.0) atomicAdd(&r.adj[i], adj_sh[i]);
  }
}

}  // namespace

/* Static shared memory (the adjoint accumulators, the cooperative rows) plus
   the staged blob can pass the 48 KB a launch gets without opting in, so
   every launch with a staged blob opts in to its dynamic size. */
template <int MODE, bool EXT, int PH, bool SMEM = true>
cudaError_t allow_dynamic_smem(size_t smem) {
  return cudaFuncSetAttribute(k_persistent<SMEM, MODE, false, EXT, PH>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int MODE, bool EXT, int PH>
cudaError_t occupancy_mode(int block, size_t smem, int* bps, bool whole) {
  if (smem > 0 && whole) {
    cudaError_t e = allow_dynamic_smem<MODE, EXT, PH>(smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        bps, k_persistent<true, MODE, false, EXT, PH>, block, smem);
  }
  if (smem > 0) {  /* staged BVH nodes of a blob read from global memory */
    cudaError_t e = allow_dynamic_smem<MODE, EXT, PH, false>(smem);
    if (e != cudaSuccess) return e;
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      bps, k_persistent<false, MODE, false, EXT, PH>, block, smem);
}

template <int MODE, bool EXT, int PH>
cudaError_t launch_mode(const GeoF32& g, const RunF32& r, int grid, int block, size_t smem,
                        cudaStream_t st) {
  if (g.stage_smem && smem > 0) {
    cudaError_t e = allow_dynamic_smem<MODE, EXT, PH>(smem);
    if (e != cudaSuccess) return e;
    k_persistent<true, MODE, false, EXT, PH><<<grid, block, smem, st>>>(g, r);
  } else {
    /* the staged BVH nodes (node_stage units) are the only dynamic part */
    const size_t ns = g.node_stage > 0 ? (size_t)g.node_stage * 16u : 0;
    if (ns > 0) {
      cudaError_t e = allow_dynamic_smem<MODE, EXT, PH, false>(ns);
      if (e != cudaSuccess) return e;
    }
    k_persistent<false, MODE, false, EXT, PH><<<grid, block, ns, st>>>(g, r);
  }
  return cudaGetLastError();
}

template <int MODE>
cudaError_t batch_occupancy_mode(int block, int* bps, bool bvh) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      bps,
      bvh ? k_persistent<false, MODE, true, true, PH_DRAIN>
          : k_persistent<false, MODE, true, false, PH_DRAIN>,
      block, 0);
}

cudaError_t persistent_batch_occupancy(int block, int* bps, bool bvh, int mode) {
  if (mode == MODE_LIST) return batch_occupancy_mode<MODE_LIST>(block, bps, bvh);
  if (mode == MODE_ADJOINT) return batch_occupancy_mode<MODE_ADJOINT>(block, bps, bvh);
  if (mode != MODE_FORWARD) return cudaErrorInvalidValue;
  return batch_occupancy_mode<MODE_FORWARD>(block, bps, bvh);
}

template <int MODE>
cudaError_t launch_batch_mode(const RunF32& r, int grid, int block, cudaStream_t st, bool bvh) {
  GeoF32 g;
  memset(&g, 0, sizeof(g));
  if (bvh) k_persistent<false, MODE, true, true, PH_DRAIN><<<grid, block, 0, st>>>(g, r);
  else k_persistent<false, MODE, true, false, PH_DRAIN><<<grid, block, 0, st>>>(g, r);
  return cudaGetLastError();
}

cudaError_t launch_persistent_batch(const RunF32& r, int grid, int block, cudaStream_t st, bool bvh,
                                    int mode) {
  if (block != kBlock) return cudaErrorInvalidConfiguration;
  if (mode == MODE_LIST) return launch_batch_mode<MODE_LIST>(r, grid, block, st, bvh);
  if (mode == MODE_ADJOINT) return launch_batch_mode<MODE_ADJOINT>(r, grid, block, st, bvh);
  if (mode != MODE_FORWARD) return cudaErrorInvalidValue;
  return launch_batch_mode<MODE_FORWARD>(r, grid, block, st, bvh);
}

/* The tail phase exists for the modes with cooperative rounds (forward,
   list, adjoint replay); a trace replay runs every flight on one lane. */
template <bool EXT, int PH>
cudaError_t occupancy_bvh(int block, size_t smem, int* bps, int mode, bool whole) {
  if (mode == MODE_LIST) return occupancy_mode<MODE_LIST, EXT, PH>(block, smem, bps, whole);
  if (mode == MODE_ADJOINT) return occupancy_mode<MODE_ADJOINT, EXT, PH>(block, smem, bps, whole);
  if (mode == MODE_TRACE) {
    if (PH == PH_TAIL) return cudaErrorInvalidValue;
    return occupancy_mode<MODE_TRACE, EXT, PH_DRAIN>(block, smem, bps, whole);
  }
  return occupancy_mode<MODE_FORWARD, EXT, PH>(block, smem, bps, whole);
}

cudaError_t persistent_occupancy(int block, size_t smem, int* bps, int mode, bool bvh, bool whole) {
  return bvh ? occupancy_bvh<true, PH_DRAIN>(block, smem, bps, mode, whole)
             : occupancy_bvh<false, PH_DRAIN>(block, smem, bps, mode, whole);
}

cudaError_t tail_occupancy(int block, size_t smem, int* bps, int mode, bool bvh, bool whole) {
  return bvh ? occupancy_bvh<true, PH_TAIL>(block, smem, bps, mode, whole)
             : occupancy_bvh<false, PH_TAIL>(block, smem, bps, mode, whole);
}

template <bool EXT, int PH>
cudaError_t launch_bvh(const GeoF32& g, const RunF32& r, int grid, int block, size_t smem,
                       cudaStream_t st, int mode) {
  if (mode == MODE_LIST) return launch_mode<MODE_LIST, EXT, PH>(g, r, grid, block, smem, st);
  if (mode == MODE_ADJOINT) return launch_mode<MODE_ADJOINT, EXT, PH>(g, r, grid, block, smem, st);
  if (mode == MODE_TRACE) {
    if (PH == PH_TAIL) return cudaErrorInvalidValue;
    return launch_mode<MODE_TRACE, EXT, PH_DRAIN>(g, r, grid, block, smem, st);
  }
  return launch_mode<MODE_FORWARD, EXT, PH>(g, r, grid, block, smem, st);
}

cudaError_t launch_persistent_fp32(const GeoF32& g, const RunF32& r, int grid, int block,
                                   size_t smem, cudaStream_t st, int mode) {
  if (block > kBlock || block % 32) return cudaErrorInvalidConfiguration;
  return g.has_ext ? launch_bvh<true, PH_DRAIN>(g, r, grid, block, smem, st, mode)
                   : launch_bvh<false, PH_DRAIN>(g, r, grid, block, smem, st, mode);
}

cudaError_t launch_tail_fp32(const GeoF32& g, const RunF32& r, int grid, int block, size_t smem,
                             cudaStream_t st, int mode) {
  if (block > kBlock || block % 32) return cudaErrorInvalidConfiguration;
  /* the tail phase reads its BVH nodes through L1 without staging the tree
     tops: its few live warps keep the nodes they walk in L1, and the staged
     copy would take that L1 from them */
  GeoF32 gt = g;
  gt.node_stage = 0;
  return g.has_ext ? launch_bvh<true, PH_TAIL>(gt, r, grid, block, smem, st, mode)
                   : launch_bvh<false, PH_TAIL>(gt, r, grid, block, smem, st, mode);
}

namespace {
/* Chunk table of a run: chunk c is particles [j, j + count) of task
   order[c / per_task], j = (c % per_task) * csz, in the queue's order. */
__global__ void k_expand_chunks(const int* __restrict__ order, int norder, int per_task, int csz,
                                int np_local, int4* __restrict__ chunks) {
  const long long n = (long long)norder * per_task;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c / per_task);
    const int j = (int)(c - (long long)k * per_task) * csz;
    chunks[c] = make_int4(__ldg(order + k), j, min(csz, np_local - j), 0);
  }
}

/* Buckets of the tail order: a quarter octave of the expected walk each. */
constexpr int kOrderBuckets = 128;
static_assert(2 * kOrderBuckets == kTailOrderExtra, "tail order histogram and cursors");

/* Tail-list slot of hand-over c (front list, then back list) and the
   bucket of its phonon's expected remaining walk.  A diffusive phonon at x
   between the baths at 0 and L takes about 1.5 x (L - x) / MFP^2 more
   flights to leave (the exit time of a random walk whose flights move it
   by 2 MFP^2 / 3 squared along x); walls and holes stretch the walk, but the
   phonons the tail phase waits for are those that rank high on it. */
__device__ __forceinline__ int order_bucket(const float4* tail, int slot, float x_len) {
  const float4 e0 = tail[(size_t)kTailUnits * slot];
  const float4 e1 = tail[(size_t)kTailUnits * slot + 1];
  const float w = fmaxf(e0.x * (x_len - e0.x), 0.0f) / (e1.w * e1.w);
  return w > 1.0f ? min(kOrderBuckets - 1, (int)(4.0f * __log2f(w))) : 0;
}

/* Hand-over c of the tail list: its slot (front list, then back list). */
__device__ __forceinline__ int tail_slot(int c, int nlong, int tail_cap) {
  return c < nlong ? c : tail_cap - 1 - (c - nlong);
}

/* One thread per hand-over: its bucket, kept in the entry's spare word
   (float4 6, z), and the bucket histogram. */
__global__ void k_order_hist(float4* __restrict__ tail, int tail_cap, const int* __restrict__ queue,
                             float x_len, int* __restrict__ hist) {
  const int nlong = min(queue[2], tail_cap);
  const int ntail = nlong + min(queue[4], tail_cap - nlong);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ntail) return;
  const int slot = tail_slot(c, nlong, tail_cap);
  const int b = order_bucket(tail, slot, x_len);
  reinterpret_cast<int*>(tail + (size_t)kTailUnits * slot + 6)[2] = b;
  atomicAdd(&hist[b], 1);
}

/* One thread per hand-over: the bucket offsets from the top bucket down
   (every block from the histogram), then the slot to its bucket's range. */
__global__ void k_order_scatter(const float4* __restrict__ tail, int tail_cap,
                                const int* __restrict__ queue, const int* __restrict__ hist,
                                int* __restrict__ cursor, int* __restrict__ order) {
  __shared__ int h[kOrderBuckets];
  const int nlong = min(queue[2], tail_cap);
  const int ntail = nlong + min(queue[4], tail_cap - nlong);
  if ((int)(blockIdx.x * blockDim.x) >= ntail) return;
  for (int b = threadIdx.x; b < kOrderBuckets; b += blockDim.x) h[b] = hist[b];
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int b = kOrderBuckets - 1; b >= 0; --b) {
      const int n = h[b];
      h[b] = run;
      run += n;
    }
  }
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ntail) return;
  const int slot = tail_slot(c, nlong, tail_cap);
  const int b = reinterpret_cast<const int*>(tail + (size_t)kTailUnits * slot + 6)[2];
  order[h[b] + atomicAdd(&cursor[b], 1)] = slot;
}
}  // namespace

cudaError_t launch_tail_order(const RunF32& r, float x_len, cudaStream_t st) {
  /* the histogram and the bucket cursors follow the order array */
  int* hist = r.tail_order + r.tail_cap;
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int) * 2 * kOrderBuckets, st);
  if (e != cudaSuccess) return e;
  const unsigned blocks = (unsigned)((r.tail_cap + 255) / 256);
  k_order_hist<<<blocks, 256, 0, st>>>(r.tail, r.tail_cap, r.queue, x_len, hist);
  k_order_scatter<<<blocks, 256, 0, st>>>(r.tail, r.tail_cap, r.queue, hist, hist + kOrderBuckets,
                                          r.tail_order);
  return cudaGetLastError();
}

cudaError_t launch_expand_chunks(const int* order, int norder, int per_task, int csz, int np_local,
                                 int4* chunks, cudaStream_t st) {
  const long long n = (long long)norder * per_task;
  if (n <= 0) return cudaSuccess;
  const long long blocks = (n + 255) / 256;
  k_expand_chunks<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(order, norder, per_task, csz,
                                                                            np_local, chunks);
  return cudaGetLastError();
}

/* Violations recorded by a bounds-checked build (PT_CHECK): count, code of
   the first (1 geometry-blob index out of range, 2 non-finite phonon state)
   and its index; reset = true clears them.  Other builds return
   cudaErrorNotSupported. */
cudaError_t check_report(long long* count, int* code, int* index, bool reset) {
#ifdef PT_CHECK
  int v[3] = {0, 0, 0};
  cudaError_t e = cudaMemcpyFromSymbol(v, g_check, sizeof(v));
  if (e != cudaSuccess) return e;
  *count = v[0];
  *code = v[1];
  *index = v[2];
  if (reset) {
    const int z[3] = {0, 0, 0};
    e = cudaMemcpyToSymbol(g_check, z, sizeof(z));
  }
  return e;
#else
  (void)count; (void)code; (void)index; (void)reset;
  return cudaErrorNotSupported;
#endif
}

}  // namespace ptg
