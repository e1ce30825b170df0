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

enum EnsLaw : int { kLawLinear = 1, kLawHertz = 2, kLawReference = 3 };
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
  // reference law: the damping coefficient of a contact with (reduced) mass
  // m is (ref_a sqrt(kn m)) / ref_b in double, rounded to float, as the
  // reference's parser forms it (KSimulationData.cpp:955-1047); ref_b = 0:
  // no damping (restitution 1)
  double ref_a, ref_b;
  double ref_m;        // (4/3) pi density: m = ref_m r^3 in double, rounded once
  // turning drum (blaze_system.rot_*): triangles and cylinders turn about
  // rot_a through rot_o at rot_w rad/s; the increment per step is (rot_cd, rot_sd)
  float3 rot_o, rot_a;
  float rot_w, rot_cd, rot_sd;
  int rot;
  // the spheres' grid of triangle candidates (EnsGeom::stri_off): the hash
  // grid, or, in a system with polyhedra, a finer one of cells of
  // 2 r_max(spheres) + skin over the same origin and extent
  float scell;
  int3 snc;
  uint32_t scell_off;
};

struct EnsWallDev {
  int kind;
  int turning;         // a cylinder or a plane that turns in place with its system's drum
                       // (coaxial cylinder, plane normal to the axis): its surface moves
  float r;             // plane: offset d (n . x = d on the plane); cylinder: radius
  float3 a, b, c;      // plane: a = unit normal into the domain; triangle: vertices;
                       // cylinder: a = point on the axis, b = unit axis
  // triangle: the unit face normal and the unit edge directions (ab, ac,
  // bc), computed in double on the host from the float vertices
  double3 n64;
  double3 e64[3];
};

// ------------------------------------------------------ accurate overlaps
// The overlap of a contact is a small difference of lengths of the size of
// the particles or of the world (|xa - xb| against ra + rb, n . x against a
// plane's offset, a distance to an axis against the cylinder radius).
// Formed in FP32 it carries ~1e-7 of the large terms, which is ~1e-3 of an
// overlap of 1e-4 r.  The overlaps are therefore formed in FP64 from the
// FP32 state: differences and products of FP32 values are exact there, and
// what rounding is left is ~1e-16 of the large terms; the result is rounded
// to FP32 once.  FP64 runs at half the FP32 rate on this GPU.  The
// translation units are compiled with -fmad=false, so the FP64 expressions
// are evaluated as written (the restatement does the same on the host).
__device__ __forceinline__ double3 d3(float3 a) {
  return make_double3((double)a.x, (double)a.y, (double)a.z);
}
__device__ __forceinline__ double3 dsub(double3 a, double3 b) {
  return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double ddot(double3 a, double3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}

// (ra + rb) - |xa - xb|
__device__ __forceinline__ float overlap_pair(float ra, float rb, float3 xa, float3 xb) {
  const double3 d = dsub(d3(xa), d3(xb));
  return (float)(((double)ra + (double)rb) - sqrt(ddot(d, d)));
}

// r - (n . p - d) for a plane n . x = d
__device__ __forceinline__ float overlap_plane(float r, float3 n, float d, float3 p) {
  return (float)(((double)r + (double)d) - ddot(d3(n), d3(p)));
}
struct EnsList {        // one copy of the neighbour list + tangential history
  uint32_t* idx;
  uint32_t* cnt;
  uint32_t* mask;       // bit k: slot k holds an active history
  float* hx;
  float* hy;
  float* hz;
  uint8_t* src;         // per slot: old slot its history came from (0xff none), or null
};

struct EnsBufs {
  StateBuf S[3];        // S[0]/S[1] ping-pong, S[2] sorted gather target
  int* pid[2];
  float4* wh[2];        // wall history, slot-major: wh[q * stride + i]
  EnsList L[2];
  int stride;           // >= n
  int cap;              // neighbour slots
  int* pat;             // polyhedra: memory position of each polyhedron id (or null)
  float* ppath;         // polyhedra: path since the last re-sort, per polyhedron id
};

// Convex polyhedra among a system's spheres (mix_device.cuh): what the
// sphere step reads about them.  A polyhedron's entry in the state carries
// minus its bounding radius in pos4.w and its polyhedron id in angv4.w (its
// path since the last re-sort is kept per polyhedron instead).  A
// sphere-polyhedron pair is evaluated once, by the polyhedron step, which
// leaves the force and torque on the sphere in the polyhedron's slot
// (sf / st[k * npoly + p], sf.w = 1 for a contact); the sphere step reads
// them through twin (per sphere slot: the polyhedron's slot that holds the
// sphere, 0xff none), which a re-sort rebuilds.
struct MixView {
  const uint8_t* twin;
  const float4* sf;
  const float4* st;
  int npoly;                 // 0: spheres only
};

struct EnsGeom {
  const EnsSysDev* sys;
  const EnsWallDev* walls;
  const uint32_t* tri_off;   // per global cell: candidate triangles (CSR), or null
  const uint32_t* tri_ids;
  const uint32_t* stri_off;  // the same on the spheres' grid (EnsSysDev::scell)
  const uint32_t* stri_ids;
  uint32_t ncell_tab;        // total hash-table entries
  int law;
  float dt, skin;
  int curved;                // 1: some wall is a cylinder or a triangle (not only planes)
  float2* rot;               // per system: (cos, sin) of the drum's turn so far
  int any_rot;               // 1: some system turns (the step compiled with the turn)
  MixView mix;
};

struct EnsCapture { float4* f; float4* t; };

// Reverse-mode tape: one arena of 32-bit words holding, per recorded
// segment, the dense blocks of its steps followed by the pool space its
// steps reserved.  The dense block of a step (n particles; word offsets):
//   pos 0, vel 4n, angv 8n (float4: the step's input state), mask 12n
//   (active histories before the step), hoff 13n (the particle's history
//   words, from TapeStep::hbase), cmask 14n (the slots the step applied its
//   law to: its contacts); 15n words rounded up to a multiple of 4.  A list
//   step (a re-sort, or the first step of a segment) also reserves, in the
//   pool at TapeStep::lblock, the list's dense arrays: cnt 0, loff n (the
//   particle's list entries, from TapeStep::lbase), perm 2n (a re-sort: old
//   index of each new position); 3n words rounded up to an even count.
// Pool space, reserved a thread block at a time: per particle and step, 3
// words per active history (slot order) then 4 per wall history (xi, wall
// id); per particle and list, 2 words per list slot: (neighbour,
// twin | src << 8), twin = the neighbour's slot that holds this particle
// (0xff: none), src = the old slot a re-sort carried the history from (0xff:
// none).  Reservations are an even number of words, so list entries are
// 8-byte aligned.
struct TapeStep {
  unsigned long long block;   // arena word of the step's dense block
  unsigned long long hbase;   // the step's history words count from here
  unsigned long long lbase;   // the list recorded for the step counts from here
  unsigned long long lblock;  // a list step: its cnt / loff / perm arrays (~0: no room)
  int rb;                     // 1 when the step re-sorted
  int lat;                    // step whose list this step used
};

struct TapeCtl {
  unsigned long long cur;     // next free arena word
  unsigned long long lim;     // reservations must end at or below this
  unsigned long long lsnap;   // cur when the current step began
  int slot;                   // the step last begun
  int lslot;                  // the step holding the current list
  int overflow;               // a reservation did not fit (nothing written)
  int pad;
};

struct EnsTape {
  uint32_t* arena;
  TapeStep* steps;            // one per step of the run
  TapeCtl* ctl;
};

__host__ __device__ constexpr unsigned long long tape_block_words(int n) {
  return ((unsigned long long)n * 15ull + 3ull) & ~3ull;
}

__host__ __device__ constexpr unsigned long long tape_list_words(int n) {
  return ((unsigned long long)n * 3ull + 1ull) & ~1ull;
}

struct TapeView {
  float4* pos;
  float4* vel;
  float4* angv;
  uint32_t* mask;
  uint32_t* hoff;
  uint32_t* cmask;
};

struct TapeList {
  uint32_t* cnt;
  uint32_t* loff;
  int32_t* perm;
};

__device__ __forceinline__ TapeList tape_list(const EnsTape& tp, unsigned long long lblock, int n) {
  uint32_t* b = tp.arena + lblock;
  const size_t m = (size_t)n;
  TapeList v;
  v.cnt = b;
  v.loff = b + m;
  v.perm = reinterpret_cast<int32_t*>(b + 2 * m);
  return v;
}

__device__ __forceinline__ TapeView tape_view(const EnsTape& tp, unsigned long long block, int n) {
  uint32_t* b = tp.arena + block;
  const size_t m = (size_t)n;
  TapeView v;
  v.pos = reinterpret_cast<float4*>(b);
  v.vel = reinterpret_cast<float4*>(b + 4 * m);
  v.angv = reinterpret_cast<float4*>(b + 8 * m);
  v.mask = b + 12 * m;
  v.hoff = b + 13 * m;
  v.cmask = b + 14 * m;
  return v;
}

// Reserves `words` consecutive pool units for the calling thread, a thread
// block at a time (one atomic per block on *cur).  Every thread of the block
// calls it; blockDim.x is a multiple of 32.  Returns the thread's first unit
// counted from `base`; ok is false (and *overflow raised) when the block's
// reservation would end past `lim` or 2^32 or more units after `base`, in
// which case nothing may be written.
__device__ __forceinline__ uint32_t tape_reserve(uint32_t words, unsigned long long* cur,
                                                 unsigned long long lim, unsigned long long base,
                                                 int* overflow, bool& ok) {
  __shared__ uint32_t s_warp[32];
  __shared__ unsigned long long s_start;
  __shared__ int s_ok;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = words;                       // inclusive scan over the warp
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) s_warp[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      const uint32_t v = s_warp[q];
      s_warp[q] = (uint32_t)tot;
      tot += v;
    }
    tot += tot & 1ull;                      // keep the cursor even
    const unsigned long long start = atomicAdd(cur, tot);
    const bool fits = start + tot <= lim && start + tot - base <= 0xffffffffull;
    if (!fits) atomicExch(overflow, 1);
    s_start = start;
    s_ok = fits ? 1 : 0;
  }
  __syncthreads();
  ok = s_ok != 0;
  return (uint32_t)(s_start - base) + s_warp[w] + (x - words);
}

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
// The same step (linear law) writing what it reads into the tape as step
// tape.ctl->slot: input state, history mask, active and wall histories.
void ens_launch_step_record(const EnsGeom& g, const EnsBufs& b, int cur, int n, StepCtl* ctl,
                            StepLink link, const EnsTape& tape, int block, cudaStream_t st);
// After a step: every turning system's (cos, sin) advanced by its increment
// and renormalised.
void ens_launch_rot_tick(const EnsGeom& g, int nsys, cudaStream_t st);
// Persistent stepping: one cooperative launch runs up to *left steps with a
// grid barrier between steps and returns at the first step that asks for a
// re-sort (ctl->rebuild_req set) or when the budget is spent, with the state
// back in S[home]; it subtracts the steps run from *left, adds them to
// *done and sets loop_h (a WHILE node's handle) to *left > 0.
struct EnsPersist {
  int* left;                           // steps still to run in this graph launch
  int* done;                           // steps run (a running count)
  int* req_step;                       // first step of the launch that asked for a re-sort
  unsigned int* bar;                   // grid barrier: arrivals, generation, abort
  cudaGraphConditionalHandle loop_h;
};
// The grid of the persistent step: every block resident (0: no fit).
int ens_persist_grid(const EnsGeom& g, int block, int n);
// coop: launch as a cooperative kernel (every block resident or no launch).
cudaError_t ens_launch_persist(const EnsGeom& g, const EnsBufs& b, int home, int n, StepCtl* ctl,
                               const int* rebuilt, const EnsPersist& p, int block, int grid,
                               bool coop, cudaStream_t st);
// One thread: the pending re-sort request into if_h, *rb = 0, the round's
// request word and barrier cleared.
void ens_launch_persist_gate(StepCtl* ctl, const EnsPersist& p, int* rb,
                             cudaGraphConditionalHandle if_h, cudaStream_t st);
void ens_launch_persist_init(const EnsPersist& p, int steps, cudaStream_t st);
// Two blocks wait at a barrier counted for three (bar: 3 zeroed words).
void ens_launch_barrier_check(unsigned int* bar, StepCtl* ctl, cudaStream_t st);
// Staged caller arrays -> state S[cur], pid = index, both list copies and
// every history cleared; flags[0] |= 1 for a radius that is not positive.
void ens_launch_pack(const float* pos3, const float* rad, const float* vel3, const float* avel3,
                     const int* sys_of, const EnsBufs& b, int cur, int* pid_dst, int n,
                     int* flags, cudaStream_t st);
void ens_launch_unpack(const EnsBufs& b, int cur, int n, const int* pid_src, float* pos3,
                       float* rad, float* vel3, float* avel3, int* sys, int* pid,
                       cudaStream_t st);

}  // namespace blaze
