// dem_common.cuh -- device-side layout of one simulation and the FP32 vector
// helpers the step kernels share.
//
// HBM layout of the particle state (structure of arrays, float4 so every
// per-particle stream is one 16-byte coalesced access):
//   pos4  = (x, y, z, radius)                 cm
//   vel4  = (vx, vy, vz, type bits)           cm/s, particle-object index
//   angv4 = (wx, wy, wz, path since rebuild)  rad/s, cm
//   pid   = int particle identity (-1 = removed), read only when re-sorting
// Three copies of the float4 streams exist: the step reads one and writes
// another (ping-pong), and a re-sort gathers into the third, which the step
// then reads instead (decided on the device, so the launch sequence is fixed
// and can be captured in a CUDA graph).
//
// Arithmetic: this translation unit family is compiled with -fmad=false and
// IEEE division/sqrt, and every expression keeps the reference's operation
// order, so FP32 results equal the reference's bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "blaze_types.h"

namespace blaze {

constexpr int kMaxTypes = 8;
constexpr int kMaxPP = 6;      // PP_Parms PP[6] per particle object
constexpr int kMaxDobj = 32;
constexpr int kMaxWallOps = 1024;

// Status bits reported by every step (bitwise OR over particles).
enum StatusBits : uint32_t {
  kStatusListOverflow = 1u,   // more candidates than neighbour slots
  kStatusOutOfGrid = 2u,      // live particle outside the hash grid
  kStatusNonFinite = 4u,      // non-finite position after integration
  kStatusTypeRange = 8u,      // particle type outside the particle-object table
  kStatusTimeout = 16u,       // a bounded device wait gave up
  kStatusPolyUndefined = 32u, // a polyhedron contact met a case the reference
                              // leaves undefined (see poly_kernels.cu)
  kStatusStaleList = 64u,     // with a skin: a particle passed half the skin
                              // between two list checks (contacts may be missed)
  kStatusCellTooSmall = 128u, // with a skin: 2 r + skin exceeds a cell edge, so the
                              // 27-cell search may miss pairs within the skin
};

// One step of the wall program: planar faces, infinite planes, a macro
// cylinder and its end caps, in the reference's world-object order
// (DEM_Kernels_Compute.cuh:312-600).
enum WallOpKind : int {
  kOpFace = 0,     // polygon face: accumulate
  kOpPlane = 1,    // infinite plane (area == -1): accumulate
  kOpCylinder = 2, // macro cylinder wall: overwrite force, accumulate torque
  kOpCapTop = 3,   // end plate: overwrite force
  kOpCapBot = 4,
};

struct WallOp {
  int kind;
  int wobj;      // the world object it came from
  int nv;        // polygon vertex count
  float area;
  float tol;
  float3 n;      // face normal / cap normal
  float3 c;      // centroid / cap centre
  float3 v[8];   // polygon vertices in vertex_Order order
  // cylinder
  float radius;
  float3 axis;   // component mask (AXIS)
  float3 cbot;   // center_bot_cap
};

struct TypeParams {
  float radius, mass, iinv;
  float3 com;        // polyhedra: centre of mass in the object file's frame
  float s_kn, s_cn, s_mus, s_muk;
  float d_kn, d_cn, d_muk;
  PP_Parms pp[kMaxPP];
};

struct DobjDev {
  float3 com, axis;
  float bound_r;
  int num_faces, num_edges;
  int num_vertex;      // vertices the polyhedron tests read (at most 8)
  int attached, translating;
  float3 velocity;
  float3 vert[8];
  Surface faces[3];
  int edge0[4], edge1[4];
};

struct SimParams {
  // grid (SimulationInfo fields)
  float3 origin, cell;
  int3 ncells;
  uint32_t ncell_tab;   // cell-table entries (largest in-grid hash + 1)
  // dynamics
  float3 gravity;
  float dt, roll_res, mill_rot_vel, drum_r;
  float tan_k;          // 0.025 / dt: the contracted law's tangential factor per (mu (ma + mb))
  int rotation, mode2d, energy_calc, is_mill, rotating_wobj, cyl_rot;
  float3 cent;
  float dobj_cyl_bound_r;
  int n_types;
  TypeParams types[kMaxTypes];
  int n_dobj;
  DobjDev dobj[kMaxDobj];
  int n_ops;
  // neighbour list
  int max_nbr;
  float skin;
};

// ----------------------------------------------------------------- float3 ops
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 vmul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }

// a / b for the three components of a by one positive, normal b, correctly
// rounded (the same numbers as three IEEE divisions), from one correctly
// rounded reciprocal y = RN(1/b) and correction steps with exact remainders
// (one fused multiply-add each): q0 = RN(a y) is within 1.5 ulp of a/b;
// q1 = RN(q0 + (a - b q0) y) is then within one ulp, and the final
// q = RN(q1 + (a - b q1) y) is a/b rounded to nearest by Markstein's theorem
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al.,
// Handbook of Floating-Point Arithmetic: with y within half an ulp of 1/b
// and q1 within an ulp of a/b, the corrected quotient is correctly rounded,
// barring underflow or overflow of the intermediate values).  A zero
// numerator keeps its sign.  Outside the range where every intermediate is
// normal and finite (b in [1e-15, 1e15], |a| in [1e-20, 1e15]: quotients
// between 1e-35 and 1e30) the IEEE division is used.  blaze_check_division
// compares it with IEEE division on the GPU.
__device__ __forceinline__ float div_rn(float a, float y, float b) {
  if (a == 0.0f) return a * y;
  if (!(fabsf(a) >= 1e-20f && fabsf(a) <= 1e15f)) return a / b;
  const float q0 = a * y;
  const float q1 = fmaf(fmaf(-q0, b, a), y, q0);
  const float r1 = fmaf(-q1, b, a);
  return r1 == 0.0f ? q1 : fmaf(r1, y, q1);
}
__device__ __forceinline__ float3 div3_rn(float3 a, float b) {
  if (!(b >= 1e-15f && b <= 1e15f)) return f3(a.x / b, a.y / b, a.z / b);
  const float y = __frcp_rn(b);
  return f3(div_rn(a.x, y, b), div_rn(a.y, y, b), div_rn(a.z, y, b));
}

}  // namespace blaze
