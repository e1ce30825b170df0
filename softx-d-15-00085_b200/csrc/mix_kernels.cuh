// mix_kernels.cuh -- launch interface of the ensemble's polyhedron kernels
// (mix_kernels.cu; the geometry and narrow phases are in mix_device.cuh).
//
// Per step, before the sphere step k_ens_step:
//   k_mix_geom        world-frame vertex offsets and face planes of every
//                     polyhedron from its orientation (FP64)
//   k_mix_poly_step   one warp per polyhedron: sphere neighbours a slot per
//                     lane (the pair's force and torque on the sphere left in
//                     the slot for the sphere step), polyhedron neighbours one
//                     pair at a time with the warp sharing the separating-axis
//                     queries, walls a candidate triangle per lane; then lane 0
//                     sums in slot order and integrates (translation, Euler's
//                     equations in the body frame, quaternion)
// and per re-sort, after the sphere list:
//   k_mix_plist       the 64-slot neighbour list of every polyhedron, its
//                     tangential histories carried by partner pid
//   k_mix_twins       per sphere slot holding a polyhedron, the polyhedron's
//                     slot that holds the sphere
#pragma once

#include "ens_kernels.cuh"
#include "mix_device.cuh"

namespace blaze {

// Staged polyhedra -> the state right after blaze_ens_set_state (memory
// order = the caller's order): pos4.w = -bounding radius, angv4.w = id,
// orientation, memory position, path and both list copies cleared.
void mix_launch_mark(const EnsBufs& b, int cur, const MixBufs& m, const int* caller_index,
                     const float4* quat, cudaStream_t st);
void mix_launch_geom(const MixBufs& m, cudaStream_t st);
void mix_launch_plist(const EnsGeom& g, const EnsBufs& b, const MixBufs& m,
                      const uint32_t* cstart, const uint32_t* cend, StepCtl* ctl,
                      const int* gate, cudaStream_t st);
// After k_mix_plist: per sphere slot holding a polyhedron, the polyhedron's
// slot that holds the sphere.
void mix_launch_twins(const EnsBufs& b, const MixBufs& m, int n, StepCtl* ctl, const int* gate,
                      cudaStream_t st);
void mix_launch_poly_step(const EnsGeom& g, const EnsBufs& b, const MixBufs& m, int cur,
                          StepCtl* ctl, StepLink link, const EnsCapture* cap, cudaStream_t st);

}  // namespace blaze
