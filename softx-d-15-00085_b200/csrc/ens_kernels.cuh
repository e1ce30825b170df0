// ens_kernels.cuh -- device layout and launch interface of the ensemble path:
// many independent sphere systems stepped together with the extended contact
// laws (linear or Hertz-Mindlin normal force, tangential history spring with
// a Coulomb cap, rolling friction).
//
// HBM layout (structure of arrays, every stream one coalesced access):
//   pos4  = (x, y, z, radius)
//   vel4  = (vx, vy, vz, bits: system id (low 24) | wall-history mask << 24)
//   angv4 = (wx, wy, wz, path since the last re-sort)
//   pid   = index of the particle in the caller's set_state arrays
// Neighbour slots (slot-major, k * stride + i) and the tangential history of
// each slot (three float arrays, same indexing) exist twice: a re-sort builds
// the other copy, carrying every active history over by partner pid.  A
// 32-bit mask per particle marks the slots whose history is active.  Wall
// history: kWallSlots float4 slots (xi, wall id bits) per particle.
//
// Arithmetic: compiled with -fmad=false and IEEE division / square root;
// the pair law is written so that the evaluation for (j, i) produces exactly
// the negated force and history of (i, j): Newton's third law holds bit for
// bit without atomics.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dem_common.cuh"
#include "dem_kernels.cuh"

namespace blaze {

constexpr int kWallSlots = 4;
constexpr uint32_t kSysBits = 24;
constexpr uint32_t kSysMask = (1u << kSysBits) - 1u;

enum EnsLaw : int { kLawLinear = 1, kLawHertz = 2 };
enum EnsWallKind : int { kWallPlane = 0, kWallTriangle = 1, kWallCylinder = 2 };

struct EnsSysDev {
  float3 origin;
  float cell;
  int3 nc;
  uint32_t cell_off;   // first global hash-table entry of this system
  float3 gravity;
  float dens43pi;      // density * 4/3 pi: m = dens43pi * r^3
  float kn, kt;        // linear law stiffnesses
  float beta2;         // linear law: 2 beta, damping c = beta2 * sqrt(m* k)
  float estar, gstar;  // Hertz-Mindlin: E*, G*
  float beta2h;        // Hertz-Mindlin: 2 sqrt(5/6) beta
  float mu, mu_w, mu_r;
  int wall0, nwall;    // planes and cylinders, tested for every particle
};

struct EnsWallDev {
  int kind;
  float r;             // plane: offset d (n . x = d on the plane); cylinder: radius
  float3 a, b, c;      // plane: a = unit normal into the domain; triangle: vertices;
                       // cylinder: a = point on the axis, b = unit axis
};

struct EnsList {        // one copy of the neighbour list + tangential history
  uint32_t* idx;
  uint32_t* cnt;
  uint32_t* mask;       // bit k: slot k holds an active history
  float* hx;
  float* hy;
  float* hz;
  uint8_t* src;         // per slot: old slot its history came from (0xff none), or null
  uint8_t* twin;        // per slot: the neighbour's slot for this particle (reverse mode)
};

struct EnsBufs {
  StateBuf S[3];        // S[0]/S[1] ping-pong, S[2] sorted gather target
  int* pid[2];
  float4* wh[2];        // wall history, slot-major: wh[q * stride + i]
  EnsList L[2];
  int stride;           // >= n
  int cap;              // neighbour slots
};

struct EnsGeom {
  const EnsSysDev* sys;
  const EnsWallDev* walls;
  const uint32_t* tri_off;   // per global cell: candidate triangles (CSR), or null
  const uint32_t* tri_ids;
  uint32_t ncell_tab;        // total hash-table entries
  int law;
  float dt, skin;
};

struct EnsCapture { float4* f; float4* t; };

void ens_launch_hash(const EnsGeom& g, const EnsBufs& b, int cur, int n, uint32_t* keys,
                     StepCtl* ctl, const int* gate, cudaStream_t st);
void ens_launch_reorder(const EnsBufs& b, int cur, int n, const uint32_t* keys,
                        const int32_t* perm, uint32_t* cstart, uint32_t* cend, uint32_t ncell_tab,
                        StepCtl* ctl, const int* gate, cudaStream_t st);
void ens_launch_nlist(const EnsGeom& g, const EnsBufs& b, int n, const int32_t* perm,
                      const uint32_t* cstart, const uint32_t* cend, StepCtl* ctl,
                      const int* gate, cudaStream_t st);
void ens_launch_epoch(StepCtl* ctl, const int* gate, cudaStream_t st);
// `block`: threads per block (64 .. kMaxStepBlock, a multiple of 32).
constexpr int kMaxStepBlock = 512;
void ens_launch_step(const EnsGeom& g, const EnsBufs& b, int cur, int n, StepCtl* ctl,
                     StepLink link, const EnsCapture* cap, int block, cudaStream_t st);
// Staged caller arrays -> state S[cur], pid = index, both list copies and
// every history cleared; flags[0] |= 1 for a radius that is not positive.
void ens_launch_pack(const float* pos3, const float* rad, const float* vel3, const float* avel3,
                     const int* sys_of, const EnsBufs& b, int cur, int* pid_dst, int n,
                     int* flags, cudaStream_t st);
void ens_launch_unpack(const EnsBufs& b, int cur, int n, const int* pid_src, float* pos3,
                       float* rad, float* vel3, float* avel3, int* sys, int* pid,
                       cudaStream_t st);

}  // namespace blaze
