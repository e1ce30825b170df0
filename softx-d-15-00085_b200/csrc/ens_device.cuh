// ens_device.cuh -- device functions shared by the ensemble's sphere step
// (ens_kernels.cu) and its polyhedron step (mix_kernels.cu): cell keys, the
// drum turn, the contact law and the sphere-wall tests.
#pragma once

#include "ens_kernels.cuh"

namespace blaze {

__device__ __forceinline__ void ens_flag(StepCtl* ctl, uint32_t bits) {
  const unsigned m = __activemask();
  const uint32_t all = __reduce_or_sync(m, bits);
  if (all && (threadIdx.x & 31) == (__ffs(m) - 1)) atomicOr(&ctl->status, all);
}

__device__ __forceinline__ int3 ens_cell(const EnsSysDev& S, float3 p) {
  int3 c;
  c.x = (int)floorf((p.x - S.origin.x) / S.cell);
  c.y = (int)floorf((p.y - S.origin.y) / S.cell);
  c.z = (int)floorf((p.z - S.origin.z) / S.cell);
  return c;
}
__device__ __forceinline__ bool ens_in(const EnsSysDev& S, int3 c) {
  return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < S.nc.x && c.y < S.nc.y && c.z < S.nc.z;
}
__device__ __forceinline__ uint32_t ens_key(const EnsSysDev& S, int3 c) {
  return S.cell_off + (uint32_t)(c.x + S.nc.x * (c.y + S.nc.y * c.z));
}
// the spheres' grid of triangle candidates
__device__ __forceinline__ int3 ens_scell(const EnsSysDev& S, float3 p) {
  int3 c;
  c.x = (int)floorf((p.x - S.origin.x) / S.scell);
  c.y = (int)floorf((p.y - S.origin.y) / S.scell);
  c.z = (int)floorf((p.z - S.origin.z) / S.scell);
  return c;
}
__device__ __forceinline__ bool ens_sin(const EnsSysDev& S, int3 c) {
  return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < S.snc.x && c.y < S.snc.y && c.z < S.snc.z;
}
__device__ __forceinline__ uint32_t ens_skey(const EnsSysDev& S, int3 c) {
  return S.scell_off + (uint32_t)(c.x + S.snc.x * (c.y + S.snc.y * c.z));
}
// v turned by the angle with cosine c and sine s about the unit axis a
// (Rodrigues): v c + (a x v) s + a (a . v) (1 - c)
__device__ __forceinline__ float3 rot_about(float3 a, float c, float s, float3 v) {
  const float3 axv = cross3(a, v);
  const float av = dot3(a, v);
  return (v * c + axv * s) + a * (av * (1.0f - c));
}

__device__ __forceinline__ float sphere_mass(const EnsSysDev& S, float r) {
  return S.dens43pi * ((r * r) * r);
}

// ------------------------------------------------------------- contact law
// kRoll = false: without the rolling-friction torque (contacts of polyhedra).
template <int kLaw, bool kRoll = true>
__device__ __forceinline__ void contact_law(const EnsSysDev& S, float mu, float3 n, float delta,
                                            float rs, float ms, float3 vrel, float3 vct,
                                            float3 wrel, float arm, float dt, float3& xi,
                                            float3& F, float3& T) {
  const float vn = dot3(vrel, n);
  float kn_e, cn, kt_e, ct;
  if (kLaw == kLawLinear) {
    kn_e = S.kn;
    kt_e = S.kt;
    cn = S.beta2 * sqrtf(ms * S.kn);
    ct = S.beta2 * sqrtf(ms * S.kt);
  } else {
    const float sq = sqrtf(rs * delta);
    const float sn = (2.0f * S.estar) * sq;
    kn_e = 0.6666667f * sn;
    kt_e = (8.0f * S.gstar) * sq;
    cn = S.beta2h * sqrtf(sn * ms);
    ct = S.beta2h * sqrtf(kt_e * ms);
  }
  const float fn = kn_e * delta - cn * vn;
  const float fc = fn > 0.0f ? fn : 0.0f;  // compressive part: friction bound
  const float3 vt = vct - dot3(vct, n) * n;
  const float xn = dot3(xi, n);
  if (xn != 0.0f) {
    const float m0 = dot3(xi, xi);
    xi = xi - xn * n;
    const float m1 = dot3(xi, xi);
    if (m1 > 0.0f) xi = xi * sqrtf(m0 / m1);
  }
  xi = xi + vt * dt;
  float3 ft = xi * (-kt_e) - vt * ct;
  const float cap = mu * fc;
  const float f2 = dot3(ft, ft);
  if (f2 > cap * cap) {
    const float s = cap / sqrtf(f2);
    ft = ft * s;
    xi = (ft + vt * ct) * (-1.0f / kt_e);
  }
  F = n * fn + ft;
  T = cross3(n * (-arm), F);
  if (kRoll && S.mu_r > 0.0f) {
    const float w2 = dot3(wrel, wrel);
    if (w2 > 0.0f) T = T + wrel * (-((S.mu_r * fc) * rs) / sqrtf(w2));
  }
}

// Closest point of triangle (a, b, c) to p by Voronoi regions of the
// vertices, edges and face (Ericson, Real-Time Collision Detection, 5.1.5).
// region: 0 face interior, 1 edge, 2 vertex; feat: the vertex (0 a, 1 b,
// 2 c) or edge (0 ab, 1 ac, 2 bc) it lies on.
__device__ __forceinline__ float3 closest_on_triangle(float3 p, float3 a, float3 b, float3 c,
                                                      int& region, int& feat) {
  const float3 ab = b - a, ac = c - a, ap = p - a;
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) { region = 2; feat = 0; return a; }
  const float3 bp = p - b;
  const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) { region = 2; feat = 1; return b; }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    region = 1;
    feat = 0;
    return a + ab * (d1 / (d1 - d3));
  }
  const float3 cp = p - c;
  const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) { region = 2; feat = 2; return c; }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    region = 1;
    feat = 1;
    return a + ac * (d2 / (d2 - d6));
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    region = 1;
    feat = 2;
    return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
  }
  const float den = 1.0f / ((va + vb) + vc);
  region = 0;
  feat = 0;
  return a + ab * (vb * den) + ac * (vc * den);
}

// Contact of a sphere (centre p, radius r) with one wall: normal from the
// wall to the centre, overlap; false when not touching.  kCurved = false
// compiles the plane test only (ensembles whose walls are all planes).
template <bool kCurved>
__device__ __forceinline__ bool wall_touch(const EnsWallDev& W, float3 p, float r, float3& n,
                                           float& delta, int& region) {
  region = 0;
  // Walls first take a conservative FP32 test (its margin is ten times the
  // FP32 rounding of the distance), so the FP64 overlap runs only near them.
  const float mag = fabsf(p.x) + fabsf(p.y) + fabsf(p.z) + fabsf(W.r);
  if (W.kind == kWallPlane) {
    if (!(dot3(W.a, p) - W.r < r + 1e-6f * mag)) return false;
    delta = overlap_plane(r, W.a, W.r, p);
    if (!(delta > 0.0f)) return false;
    n = W.a;
    return true;
  }
  if constexpr (!kCurved) return false;
  if (W.kind == kWallCylinder) {
    {
      const float3 v = p - W.a;
      if (!(len3(v - dot3(v, W.b) * W.b) + r > W.r - 1e-6f * (mag + 2.0f * W.r))) return false;
    }
    // rad = v - (v . b) b with v = p - a, in double
    const double3 v = dsub(d3(p), d3(W.a)), b = d3(W.b);
    const double vb = ddot(v, b);
    const double3 rad = make_double3(v.x - vb * b.x, v.y - vb * b.y, v.z - vb * b.z);
    const double rho = sqrt(ddot(rad, rad));
    delta = (float)(((double)r + rho) - (double)W.r);
    if (!(delta > 0.0f) || !(rho > 0.0)) return false;
    const float rinv = (float)(-1.0 / rho);
    n = f3((float)rad.x * rinv, (float)rad.y * rinv, (float)rad.z * rinv);
    return true;
  }
  int feat;
  const float3 q = closest_on_triangle(p, W.a, W.b, W.c, region, feat);
  const float3 d = p - q;
  const float d2 = dot3(d, d);
  if (!(d2 < r * r)) return false;
  if (region == 0) {
    // face: the signed distance (p - a) . n, n the unit normal in double
    const double s = ddot(dsub(d3(p), d3(W.a)), W.n64);
    delta = (float)((double)r - fabs(s));
    if (!(delta > 0.0f) || !(s != 0.0)) return false;
    const float sg = s < 0.0 ? -1.0f : 1.0f;
    n = f3((float)W.n64.x * sg, (float)W.n64.y * sg, (float)W.n64.z * sg);
    return true;
  }
  // vertex: p - v; edge: p - v0 less its part along the unit edge e
  const float3 v0 = region == 2 ? (feat == 0 ? W.a : (feat == 1 ? W.b : W.c))
                                : (feat == 2 ? W.b : W.a);
  double3 pv = dsub(d3(p), d3(v0));
  if (region == 1) {
    const double3 e = W.e64[feat];
    const double t = ddot(pv, e);
    pv = make_double3(pv.x - t * e.x, pv.y - t * e.y, pv.z - t * e.z);
  }
  const double dist = sqrt(ddot(pv, pv));
  delta = (float)((double)r - dist);
  if (!(delta > 0.0f) || !(dist > 0.0)) return false;
  const float dinv = (float)(1.0 / dist);
  n = f3((float)pv.x * dinv, (float)pv.y * dinv, (float)pv.z * dinv);
  return true;
}

}  // namespace blaze
