// ens_adjoint.cuh -- reverse mode of the ensemble step (linear law with
// tangential history and Coulomb cap, plane walls, no rolling friction).
//
// A forward segment is recorded step by step into a tape; the reverse sweep
// then walks the tape backwards.  Per step the tape keeps what the step
// read: its input state (after a re-sort), the neighbour list with masks
// and histories before the step, the wall history, and for a re-sort step
// the permutation and the old slot of each carried history.
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

struct EnsTape {
  int K;                // steps the tape holds
  int* rb;              // per step: 1 when the step re-sorted
  int32_t* perm;        // per step, n: old index of each new position
  uint8_t* src;         // per step, cap x n: carried history's old slot
  float4* pos;          // per step, n: input state
  float4* vel;
  float4* angv;
  uint32_t* idx;        // per step, cap x n: the list the step used
  uint32_t* cnt;        // per step, n
  uint32_t* mask;       // per step, n: active histories before the step
  float* hx;            // per step, cap x n: histories before the step
  float* hy;
  float* hz;
  float4* wh;           // per step, kWallSlots x n: wall histories before the step
  uint8_t* twin;        // per step, cap x n: the neighbour's slot for this particle
};

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
  float4* Tb;
  float4* px;           // per list slot (cap x n): the share of a contact's
  float4* pv;           // cotangent that goes to the neighbour's state
  float4* pw;
  float* th;            // per position: kn, kt, 2 beta, mu, mu_wall cotangents (n x 5)
};

// Copy what step `t` of the tape needs (after the step's re-sort, before the
// step kernel) from the ensemble's buffers; `rebuilt` is the device flag of
// the step, `perm` the sort result.
void adj_launch_snap(const EnsTape& tp, int t, const EnsBufs& b, int cur, int n,
                     const StepCtl* ctl, const int* rebuilt, const int32_t* perm,
                     cudaStream_t st);
// The same with the tape step read from *slot on the device, followed by a
// one-thread kernel that advances *slot (so a captured graph can record into
// successive tape steps).
void adj_launch_snap_slot(const EnsTape& tp, int* slot, const EnsBufs& b, int cur, int n,
                          const StepCtl* ctl, const int* rebuilt, const int32_t* perm,
                          cudaStream_t st);
// For every slot of the current list, the neighbour's slot that holds this
// particle (0xff if the neighbour's list overflowed); `gate` as in the
// re-sort kernels.
void adj_launch_twin(const EnsBufs& b, int n, const StepCtl* ctl, const int* gate,
                     cudaStream_t st);
// Reverse of tape step t, which used the list stored at tape step tl (the
// last re-sort step <= t, or the tape's first step): cotangents after the
// step (gx..gW) -> before it (ix..iW), law-constant cotangents added to th.
void adj_launch_step(const EnsGeom& g, const EnsTape& tp, int t, int tl, int n, int cap,
                     const AdjBufs& a, cudaStream_t st);
// Reverse of the re-sort of tape step t: cotangents before the step (ix..iW,
// sorted order) -> after the previous step (gx..gW, order before the sort).
void adj_launch_unsort(const EnsTape& tp, int t, int n, int cap, const AdjBufs& a,
                       cudaStream_t st);

// Host-layout (3 floats per particle) cotangents to and from float4;
// src == nullptr gives zeros.
void adj_launch_f3_to_f4(const float* src, float4* dst, int n, cudaStream_t st);
void adj_launch_f4_to_f3(const float4* src, float* dst, int n, cudaStream_t st);
// out[5 s + c] = sum over the particles [off[s], off[s + 1]) of th[5 i + c],
// in FP64, in particle order.
void adj_launch_sum_constants(const float* th, const int* off, int nsys, double* out,
                              cudaStream_t st);

}  // namespace blaze
