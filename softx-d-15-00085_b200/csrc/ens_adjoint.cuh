// ens_adjoint.cuh -- reverse mode of the ensemble step (linear law with
// tangential history and Coulomb cap, plane walls, no rolling friction).
//
// A forward segment is recorded step by step into a tape (EnsTape,
// ens_kernels.cuh); the reverse sweep then walks the tape backwards.  Per
// step the tape keeps what the step read: its input state (after a
// re-sort), the history mask with the active histories and the wall
// histories; at a list step the list with the twin slots, and at a re-sort
// step the permutation and the old slot of each carried history.
//
// The reverse of a step is the exact derivative of the forward arithmetic
// on the branch each contact took (contact or not, stick or slip, history
// turned into the tangent plane or not): active-branch derivatives at
// contact onset and stick/slip switches.  Every kernel gathers: a particle
// collects the cotangent its neighbours' contacts send it by evaluating the
// same pair from their side, so no atomics are used.
#pragma once

#include "ens_kernels.cuh"

namespace blaze {

struct AdjBufs {        // cotangents, all in the memory order of the step they belong to
  float4* gx;           // of the positions (after the step being reversed)
  float4* gv;
  float4* gw;
  float4* gH;           // of the list histories, cap x n
  float4* gW;           // of the wall histories, kWallSlots x n
  float4* ix;           // the same, before the step (double buffers)
  float4* iv;
  float4* iw;
  float4* iH;
  float4* iW;
  float4* Fb;           // host cotangent stage (the force cotangents stay in registers)
  float4* px;           // per list slot (cap x n): the share of a contact's
  float4* pv;           // cotangent that goes to the neighbour's state
  float4* pw;
  float* th;            // per position: kn, kt, 2 beta, mu, mu_wall cotangents (n x 5)
};

// Recording, all on the device (so that a captured graph can record into
// successive steps):
//   adj_launch_seg_start  a segment of `len` steps from step slot0: dense
//                         blocks from arena word `origin` (`stride` words
//                         each), pool space after them up to `lim`;
//   adj_launch_list       record the current list (count, entries, twins;
//                         with `resorted`, carried-history slots and the
//                         permutation `perm`) as the list of the step about
//                         to begin; `gate` as in the re-sort kernels;
//   adj_launch_tick       begin the next step: re-sort flag (*rebuilt), list
//                         step, history base;
//   ens_launch_step_record  the step itself, writing what it reads.
void adj_launch_seg_start(const EnsTape& tp, int slot0, int len, unsigned long long origin,
                          unsigned long long stride, unsigned long long lim, cudaStream_t st);
void adj_launch_list(const EnsBufs& b, const EnsTape& tp, int n, const StepCtl* ctl,
                     const int* gate, int resorted, const int32_t* perm, cudaStream_t st);
void adj_launch_tick(const EnsTape& tp, const int* rebuilt, cudaStream_t st);
// Reverse of tape step t: cotangents after the step (gx..gW) -> before it
// (ix..iW), law-constant cotangents added to th.  Only the history and wall
// slots that the reverse of the step before reads are written: slot k of
// particle i where the step's input mask has bit k, wall slots of the
// step's input wall mask.
void adj_launch_step(const EnsGeom& g, const EnsTape& tp, int t, int n, const AdjBufs& a,
                     cudaStream_t st);
// Reverse of the re-sort of tape step t: cotangents before the step (ix..iW,
// sorted order) -> after the previous step (gx..gW, order before the sort).
// Every history slot the step before reads was carried by the re-sort (its
// contacts are all inside the new list's range), so the scatter covers them.
void adj_launch_unsort(const EnsTape& tp, int t, int n, const AdjBufs& a, cudaStream_t st);

// Host-layout (3 floats per particle) cotangents to and from float4;
// src == nullptr gives zeros.
void adj_launch_f3_to_f4(const float* src, float4* dst, int n, cudaStream_t st);
void adj_launch_f4_to_f3(const float4* src, float* dst, int n, cudaStream_t st);
// out[5 s + c] = sum over the particles [off[s], off[s + 1]) of th[5 i + c],
// in FP64 (a fixed reduction tree per system, so repeated calls agree).
void adj_launch_sum_constants(const float* th, const int* off, int nsys, double* out,
                              cudaStream_t st);

}  // namespace blaze
