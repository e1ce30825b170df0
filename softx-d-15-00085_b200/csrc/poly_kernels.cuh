// poly_kernels.cuh -- convex polyhedra on the reference path.
//
// A polyhedral particle is its bounding sphere in the broad phase (the
// sphere path's hash, sort, reorder and contact-list kernels run unchanged),
// plus, per step:
//   k_poly_geom  world-frame vertices and face planes of every particle,
//                written once (the reference rotates particle B again for
//                every pair, DEM_Kernels_Compute.cuh:820);
//   k_poly_step  particle-particle narrow phase and law, world objects and
//                symplectic Euler with the quaternion update, fused, one
//                thread per particle, gather only.
// Orientations live beside P_ID (two copies selected by the re-sort count),
// gathered by the re-sort and updated in place by the step.
#pragma once

#include "dem_kernels.cuh"

namespace blaze {

constexpr int kPolyMaxV = 32;   // POBJ::Local_Vertex[32]
constexpr int kPolyMaxF = 32;   // POBJ::face[32]
constexpr int kPolyMaxE = 32;   // POBJ::edge[32]
constexpr int kPolyFaceV = 8;   // Surface::vertex_Order[8]

// One particle object in its body frame (KSimulationObjects.h:272-304),
// validated and repacked by the host.
struct PolyShape {
  int nv, nf, ne, pad;
  float4 vert[kPolyMaxV];          // Local_Vertex
  float4 fnorm[kPolyMaxF];         // face normal
  float4 fcent[kPolyMaxF];         // face centroid - COM
  float farea[kPolyMaxF];
  int fnv[kPolyMaxF];              // vertices of each face
  uint8_t ford[kPolyMaxF][kPolyFaceV];  // vertex_Order
  uint8_t edge[kPolyMaxE][2];      // point_vindex
  float inertia[9];                // InertiaT as the host scaled it (main.cpp:622-626)
  float com[3];
};

// World-frame geometry of every particle, rebuilt each step: particle i's
// vertices at vert[i * kv ...], face normals and centroids at
// fnorm/fcent[i * kf ...].
struct PolyGeom {
  float4* vert;
  float4* fnorm;
  float4* fcent;
  int kv, kf;
};

void launch_poly_geom(const PolyShape* shapes, PolyGeom g, const StateBuf& in_plain,
                      const StateBuf& in_sorted, const OrderBuf& ob, int n_max, int rotation,
                      const StepCtl* ctl, const int* rebuilt, cudaStream_t st);

void launch_poly_step(const SimParams* dp, const PolyShape* shapes, PolyGeom g,
                      const WallOp* ops, const StateBuf& in_plain, const StateBuf& in_sorted,
                      const StateBuf& out, const OrderBuf& ob, int n_max, NbrList nl,
                      StepCtl* ctl, StepLink link, const ForceCapture* cap, cudaStream_t st);

}  // namespace blaze
