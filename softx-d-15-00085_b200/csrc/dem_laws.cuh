// dem_laws.cuh -- the reference's contact laws and point-in-polygon test as
// FP32 device functions, shared by the sphere and polyhedron step kernels.
// Every expression keeps the reference's operation order (the translation
// units that include this file are compiled with -fmad=false); a vector
// divided by a scalar goes through div3_rn (dem_common.cuh), which gives
// the IEEE quotients bit for bit.
#pragma once

#include "dem_common.cuh"

namespace blaze {

struct Forces { float3 trans, torque; };

// The reference's contact test |xa - xb| - (ra + rb) < 0
// (Collision_Detection_BroadPhase.cuh:376, len3 then a subtraction), decided
// without the square root wherever that is exact.  With d2 formed as len3
// forms it, the test is RN(sqrt(d2)) < sr (the difference of two distinct
// floats never rounds to zero).  With s2 = RN(sr^2): d2 < RN(s2 (1 - 2^-20))
// implies sqrt(d2) < sr (1 - 2^-22), so RN(sqrt(d2)) < sr; d2 > RN(s2 (1 +
// 2^-20)) implies sqrt(d2) > sr (1 + 2^-23), so RN(sqrt(d2)) > sr (each
// rounding moves a value by at most 2^-24 of itself while s2 is normal).
// In between, and for NaN or tiny radii, the IEEE square root decides.
__device__ __forceinline__ bool touches(float3 rel, float sr) {
  const float d2 = dot3(rel, rel);
  const float s2 = sr * sr;
  if (s2 >= 1e-30f) {
    if (d2 < s2 * (1.0f - 0x1p-20f)) return true;
    if (d2 > s2 * (1.0f + 0x1p-20f)) return false;
  }
  return sqrtf(d2) - sr < 0.0f;
}


// Energy tallies (SimulationInfo::EnergyCalc): a law given `e` stores there
// the value the reference adds to its tally for this contact (normal
// dissipation |Fdiss| |Vn| dt, unless the force was attractive, plus the
// tangential |Ft| |Vt| dt), in the reference's operation order; the caller
// sums them.  e == nullptr (the default) computes forces only.

// Collision_Response_Particle_Particle, Collision_Response.cuh:374-494.
// kSpin = false is the spin-free form used when
// rotation is off and every angular velocity is exactly zero: then
// v + cross(0, R) equals v up to the sign of an exact zero, so the forces
// are the same numbers.
// The tangential force's factor (((0.5 (m_a + m_b)) / dt) 0.05) mu_k, which
// depends on the two particle types only; law_pp_pre takes it precomputed.
__device__ __forceinline__ float tangential_prefactor(const SimParams& P, const PP_Parms& pp,
                                                      float ma, float mb) {
  return (((0.50f * (ma + mb)) / P.dt) * 0.050f) * pp.Fric_kinetic;
}

template <bool kSpin>
__device__ __forceinline__ Forces law_pp_pre(const SimParams& P, float3 rvel, float3 n, float pen,
                                             float3 ra, float3 rb, float3 wa, float3 wb,
                                             const PP_Parms& pp, float3 va, float3 vb,
                                             float tan_pre, float* e = nullptr) {
  Forces F;
  const float3 vn = dot3(rvel, n) * n;
  const float fn = pp.Kn * pen;
  const float3 fdiss = pp.Cn * vn;
  F.trans = fn * n - fdiss;
  // the non-symmetric path evaluates every contact from both sides: half each
  float en = 0.0f;
  if (e && dot3(vn, vn) > 0.0f) en = ((0.50f * len3(fdiss)) * len3(vn)) * P.dt;
  const float3 vcpa = kSpin ? va + cross3(wa, ra) : va;
  const float3 vcpb = kSpin ? vb + cross3(wb, rb) : vb;
  const float3 vcpna = dot3(vcpa, n) * n;
  const float3 vcpnb = dot3(vcpb, n) * n;
  const float3 vt = (vcpa - vcpna) - (vcpb - vcpnb);
  float mag = dot3(vt, vt);
  float3 ft = f3(0.0f, 0.0f, 0.0f);
  if (mag > 0.0f) {
    mag = sqrtf(mag);
    float velf = dot3(rvel, rvel);
    if (velf > 0) velf = sqrtf(velf);
    else velf = 1.0f;
    const float tan_f = tan_pre * (mag / velf);
    ft = (-1.0f * tan_f) * div3_rn(vt, mag);
    if (e) en = en + ((len3(ft) * mag) * P.dt);
  }
  if (e) *e = en;
  F.trans = F.trans + ft;
  F.torque = (kSpin && P.rotation) ? cross3(ra, F.trans) : f3(0.0f, 0.0f, 0.0f);
  return F;
}

template <bool kSpin>
__device__ __forceinline__ Forces law_pp(const SimParams& P, float3 rvel, float3 n, float pen,
                                         float3 ra, float3 rb, float3 wa, float3 wb,
                                         const PP_Parms& pp, float3 va, float3 vb, float ma,
                                         float mb, float* e = nullptr) {
  return law_pp_pre<kSpin>(P, rvel, n, pen, ra, rb, wa, wb, pp, va, vb,
                           tangential_prefactor(P, pp, ma, mb), e);
}

// The reference's particle-particle law (law_pp_pre) in contracted form,
// for runs that ask for agreement within a tolerance instead of bit for bit:
// fused multiply-adds, an approximate reciprocal square root, and the
// tangential force as -(tan_pre / |v_rel|) v_t, which is the reference's
// -(tan_pre |v_t| / |v_rel|) (v_t / |v_t|) without forming |v_t|.  The
// normal force uses the caller's penetration unchanged (it carries the
// cancellation of |xa - xb| - (ra + rb), so it is formed as the reference
// forms it).  Differs from law_pp_pre by a few ulp of the force's terms.
template <bool kSpin>
__device__ __forceinline__ Forces law_pp_fast(const SimParams& P, float3 rvel, float3 n,
                                              float pen, float3 ra, float3 rb, float3 wa,
                                              float3 wb, const PP_Parms& pp, float3 va,
                                              float3 vb, float tan_pre) {
  Forces F;
  const float vrn = fmaf(rvel.x, n.x, fmaf(rvel.y, n.y, rvel.z * n.z));
  // Kn pen n - Cn (v_rel . n) n
  const float fnt = fmaf(-pp.Cn, vrn, pp.Kn * pen);
  float3 dv = rvel;
  float dvn = vrn;
  if (kSpin) {
    // (va + wa x ra) - (vb + wb x rb)
    dv = f3(rvel.x + fmaf(wa.y, ra.z, -wa.z * ra.y) - fmaf(wb.y, rb.z, -wb.z * rb.y),
            rvel.y + fmaf(wa.z, ra.x, -wa.x * ra.z) - fmaf(wb.z, rb.x, -wb.x * rb.z),
            rvel.z + fmaf(wa.x, ra.y, -wa.y * ra.x) - fmaf(wb.x, rb.y, -wb.y * rb.x));
    dvn = fmaf(dv.x, n.x, fmaf(dv.y, n.y, dv.z * n.z));
  }
  // v_t = dv - (dv . n) n
  const float3 vt = f3(fmaf(-dvn, n.x, dv.x), fmaf(-dvn, n.y, dv.y), fmaf(-dvn, n.z, dv.z));
  const float vt2 = fmaf(vt.x, vt.x, fmaf(vt.y, vt.y, vt.z * vt.z));
  float3 f = n * fnt;
  if (vt2 > 0.0f) {
    const float v2 = fmaf(rvel.x, rvel.x, fmaf(rvel.y, rvel.y, rvel.z * rvel.z));
    const float k = -tan_pre * (v2 > 0.0f ? rsqrtf(v2) : 1.0f);
    f = f3(fmaf(k, vt.x, f.x), fmaf(k, vt.y, f.y), fmaf(k, vt.z, f.z));
  }
  F.trans = f;
  F.torque = (kSpin && P.rotation) ? f3(fmaf(ra.y, f.z, -ra.z * f.y), fmaf(ra.z, f.x, -ra.x * f.z),
                                        fmaf(ra.x, f.y, -ra.y * f.x))
                                   : f3(0.0f, 0.0f, 0.0f);
  return F;
}

// Collision_Response_Particle_StaticSurface, Collision_Response.cuh:4-109
__device__ __forceinline__ Forces law_static_surface(const SimParams& P, float3 pvel, float3 n,
                                                     float pen, float3 r, float3 w,
                                                     const TypeParams& T, float* e = nullptr) {
  Forces F;
  const float3 vn = dot3(pvel, n) * n;
  const float fn = T.s_kn * pen;
  const float3 fdiss = T.s_cn * vn;
  F.trans = fn * n - fdiss;
  const float3 fdir = div3_rn(F.trans, len3(F.trans));
  float en = 0.0f;
  if (dot3(fdir, n) < 0) F.trans = fn * n;
  else if (e && dot3(vn, vn) > 0.0f) en = (len3(fdiss) * len3(vn)) * P.dt;
  float3 vt = pvel - vn;
  if (P.rotation) vt = vt + cross3(w, r);
  float mag = dot3(vt, vt);
  float3 ft = f3(0.0f, 0.0f, 0.0f);
  if (mag > 0.0f) {
    mag = sqrtf(mag);
    float velf = dot3(pvel, pvel);
    if (velf > 0) velf = sqrtf(velf);
    else velf = 1.0f;
    const float tan_f = (0.050f * (T.mass / P.dt)) * (T.s_mus * (mag / velf));
    ft = (-1.0f * tan_f) * div3_rn(vt, mag);
    if (e) en = en + ((len3(ft) * mag) * P.dt);
  }
  if (e) *e = en;
  F.trans = F.trans + ft;
  F.torque = P.rotation ? cross3(r, F.trans) : f3(0.0f, 0.0f, 0.0f);
  return F;
}

// Collision_Response_Particle_MovingSurface, Collision_Response.cuh:116-233
template <bool kSpin>
__device__ __forceinline__ Forces law_moving_surface(const SimParams& P, float3 n, float pen,
                                                     float3 r, float3 w, const TypeParams& T,
                                                     float3 va, float3 vs, float* e = nullptr) {
  Forces F;
  const float3 rvel = va - vs;
  const float3 vn = dot3(rvel, n) * n;
  const float fn = T.s_kn * pen;
  const float3 fdiss = T.s_cn * vn;
  F.trans = fn * n - fdiss;
  const float3 fdir = div3_rn(F.trans, len3(F.trans));
  float en = 0.0f;
  if (dot3(fdir, n) < 0) F.trans = fn * n;
  else if (e && dot3(vn, vn) > 0.0f) en = (len3(fdiss) * len3(vn)) * P.dt;
  const float3 vcpa = kSpin ? va + cross3(w, r) : va;
  const float3 vcpna = dot3(vcpa, n) * n;
  const float3 vt = (vcpa - vcpna) - (vs - dot3(vs, n) * n);
  float mag = dot3(vt, vt);
  float3 ft = f3(0.0f, 0.0f, 0.0f);
  if (mag > 0.0f) {
    mag = sqrtf(mag);
    float velf = dot3(rvel, rvel);
    if (velf > 0) velf = sqrtf(velf);
    else velf = 1.0f;
    const float tan_f = T.s_muk * (mag / velf);
    ft = (((-1.0f * tan_f) * div3_rn(vt, mag)) * (T.mass / P.dt)) * 0.050f;
    if (e) en = en + ((len3(ft) * mag) * P.dt);
  }
  if (e) *e = en;
  F.trans = F.trans + ft;
  F.torque = P.rotation ? cross3(r, F.trans) : f3(0.0f, 0.0f, 0.0f);
  return F;
}

// Collision_Response_Particle_VolumeObject, Collision_Response.cuh:241-363,
// with the zero object spin and lever the caller passes
// (DEM_Kernels_Compute.cuh:206-216).
template <bool kSpin>
__device__ __forceinline__ Forces law_volume(const SimParams& P, float3 n, float pen, float3 r,
                                             float3 w, const TypeParams& T, float3 va,
                                             float3 vobj, float* e = nullptr) {
  Forces F;
  const float3 rvel = va - vobj;
  const float3 vn = dot3(rvel, n) * n;
  const float fn = T.d_kn * pen;
  const float3 fdiss = T.d_cn * vn;
  F.trans = fn * n - fdiss;
  const float3 fdir = div3_rn(F.trans, len3(F.trans));
  float en = 0.0f;
  if (dot3(fdir, n) < 0) F.trans = fn * n;
  else if (e && dot3(vn, vn) > 0.0f) en = (len3(fdiss) * len3(vn)) * P.dt;
  const float3 z = f3(0.0f, 0.0f, 0.0f);
  const float3 vcpa = kSpin ? va + cross3(w, r) : va;
  const float3 vcpb = vobj + cross3(z, z);
  const float3 vt = (vcpa - dot3(vcpa, n) * n) - (vcpb - dot3(vcpb, n) * n);
  float mag = dot3(vt, vt);
  float3 ft = z;
  if (mag > 0.0f) {
    mag = sqrtf(mag);
    float velf = dot3(rvel, rvel);
    if (velf > 0) velf = sqrtf(velf);
    else velf = 1.0f;
    const float tan_f = (0.050f * (T.mass / P.dt)) * (T.d_muk * (mag / velf));
    ft = (-1.0f * tan_f) * div3_rn(vt, mag);
    if (e) en = en + ((len3(ft) * mag) * P.dt);
  }
  if (e) *e = en;
  F.trans = F.trans + ft;
  F.torque = P.rotation ? cross3(r, F.trans) : z;
  return F;
}

// Collision_Response_EndPlate_Particle, Collision_Response.cuh:504-526
__device__ __forceinline__ float3 law_end_plate(float3 rvel, float3 n, float pen,
                                                const TypeParams& T) {
  const float3 vn = dot3(rvel, n) * n;
  const float3 fdiss = T.s_cn * vn;
  const float fn = T.s_kn * pen;
  return fn * n - fdiss;
}

// is_PointOnSurface, Utilities.cuh:20-53
__device__ __forceinline__ bool point_on_polygon(int nv, const float3* v, float3 pt, float sarea,
                                                 float tol) {
  float area = 0.0f;
  for (int i = 0; i < nv - 1; ++i) {
    const float3 v1 = pt - v[i];
    const float3 v2 = pt - v[i + 1];
    area = area + 0.500000f * len3(cross3(v1, v2));
  }
  const float3 v1 = pt - v[nv - 1];
  const float3 v2 = pt - v[0];
  area = area + 0.500000f * len3(cross3(v1, v2));
  return (fabsf(area - sarea) / sarea) * 100.0000f <= tol;
}

// is_PointOnSurface over vertices addressed through vertex_Order.
__device__ __forceinline__ bool point_on_indexed_polygon(int nv, const float3* v, const int* order,
                                                         float3 pt, float sarea, float tol) {
  float area = 0.0f;
  for (int i = 0; i < nv - 1; ++i) {
    const float3 v1 = pt - v[order[i] & 7];
    const float3 v2 = pt - v[order[i + 1] & 7];
    area = area + 0.500000f * len3(cross3(v1, v2));
  }
  const float3 v1 = pt - v[order[nv - 1] & 7];
  const float3 v2 = pt - v[order[0] & 7];
  area = area + 0.500000f * len3(cross3(v1, v2));
  return (fabsf(area - sarea) / sarea) * 100.0000f <= tol;
}

__device__ __forceinline__ float3 drum_velocity(const SimParams& P, float3 cp) {
  return cross3(f3(0.0f, 0.0f, -P.mill_rot_vel), cp - f3(P.drum_r, P.drum_r, 0.0f));
}

}  // namespace blaze
