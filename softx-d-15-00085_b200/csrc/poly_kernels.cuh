// poly_kernels.cuh -- convex polyhedra on the reference path.
//
// A polyhedral particle is its bounding sphere in the broad phase (the
// sphere path's hash, sort, reorder and contact-list kernels run unchanged),
// plus, per step:
//   k_poly_geom  world-frame vertices and face planes of every particle,
//                written once (the reference rotates particle B again for
//                every pair, DEM_Kernels_Compute.cuh:820);
//   k_poly_sep, k_poly_vf, k_poly_ee
//                the narrow phase in three passes over the neighbour slots
//                (separating planes per slot, vertex-face per queued slot,
//                edge-edge per queued slot with a warp each);
//   k_poly_step  particle-particle law over the contacts found, volume and
//                world objects, symplectic Euler with the quaternion update,
//                one thread per particle, gather only.
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
  float rmax;                      // upper bounds on the vertices' distance from the
  float emax;                      // centre and on the edge lengths (edge-edge pruning)
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

// Narrow-phase state of one step, per neighbour slot (slot = k * stride + i):
// the verdict of the passes and, for a contact, its normal, depth and point.
struct PolyPairs {
  uint8_t* status;    // cap x stride: 0 none, 1 vertex test pending, 2 contact, 3 edge test pending
  uint8_t* hint;      // cap x stride: the face that last separated the slot's pair
                      // (bit 7: a face of the neighbour), 0xff none
  float4* con;        // 2 x cap x stride: (normal, depth), (contact point, 0)
  uint32_t* qv;       // slots queued for the vertex-face test
  uint32_t* qe;       // slots queued for the edge-edge test
  int* counts;        // [0] vertex-face queue length, [1] edge-edge queue length,
                      // [2] filled neighbour slots (NbrList::flat_n)
  int grid_s, grid_v, grid_e;  // blocks of the three passes (persistent grids)
};

void launch_poly_geom(const PolyShape* shapes, PolyGeom g, const StateBuf& in_plain,
                      const StateBuf& in_sorted, const OrderBuf& ob, int n_max, int rotation,
                      const StepCtl* ctl, const int* rebuilt, cudaStream_t st);

// The three narrow-phase passes (separating planes, vertex-face, edge-edge)
// over the step's neighbour slots; returns the number of kernel launches.
int launch_poly_pairs(const SimParams* dp, const PolyShape* shapes, PolyGeom g,
                      const StateBuf& in_plain, const StateBuf& in_sorted, int n_max, NbrList nl,
                      StepCtl* ctl, const int* rebuilt, PolyPairs pp, cudaStream_t st);

// eb: when not null, also the energy-tally values per particle (as
// launch_step).
void launch_poly_step(const SimParams* dp, const PolyShape* shapes, PolyGeom g,
                      const WallOp* ops, const StateBuf& in_plain, const StateBuf& in_sorted,
                      const StateBuf& out, const OrderBuf& ob, int n_max, NbrList nl,
                      PolyPairs pp, StepCtl* ctl, StepLink link, const ForceCapture* cap,
                      double* eb, cudaStream_t st);

}  // namespace blaze
