// dem_kernels.cuh -- launch interface of the per-step kernels.
#pragma once

#include "dem_common.cuh"

namespace blaze {

struct StateBuf {
  float4* pos;    // (x, y, z, radius)
  float4* vel;    // (vx, vy, vz, type bits)
  float4* angv;   // (wx, wy, wz, path since rebuild)
};

// Arrays that only change order when the particles are re-sorted: two
// copies, selected by the parity of StepCtl::epoch (the re-sort count).
struct OrderBuf {
  int* pid[2];
  int* lift[2];      // volume-object contact type (Contact_Info.cont_type)
  float4* ornt[2];   // polyhedra: orientation (w, x, y, z); null for spheres
};

struct ForceCapture {   // optional per-particle force dump (parity tests)
  float* f_pp; float* t_pp; float* f_w; float* t_w; float* f_l; float* t_l;
};

struct StepCtl {        // device words the step pipeline communicates through
  int rebuild_req;      // set by the step (or a removal) when the list must be rebuilt
  int rebuilt;          // 1 while the current step consumes a fresh re-sort
  uint32_t status;      // StatusBits of the current run
  int epoch;            // number of re-sorts so far (selects OrderBuf copies)
  int n_cur;            // live particles (removed ones sit at the end)
  int pending_dead;     // removed since the last re-sort
  int killed_total;
  int exact_blocks;     // with a skin: blocks of steps run in the exact mode so far
  uint32_t* chk;        // with a skin: kChkSlots maxima of path, then of speed (float
                        // bits, one per 128-byte line), recorded at the step before a check
  int exact;            // with a skin: 1 = this block of steps checks before every step
  int gate_r;           // the gate's re-sort decision, for the first IF of a graph body
};

struct NbrList {
  uint32_t* idx;        // slot-major: idx[k * stride + i]
  uint32_t* cnt;
  int stride;           // >= n_max
  int cap;
  uint32_t* flat;       // optional: every filled slot k * stride + i, particle by particle
  int* flat_n;          // entries in `flat` (reset before each rebuild)
};

// How a step learns whether it consumes a fresh re-sort, and how it asks for
// the next one: through StepCtl (plain stepping) or, inside a CUDA graph,
// through the IF-node condition of the next step.
struct StepLink {
  const int* rebuilt;                  // nonzero: read the sorted buffer
  cudaGraphConditionalHandle next_h;   // next step's IF condition (graph)
  int has_next_h;                      // 0: request through StepCtl::rebuild_req
  int check_next;                      // with a skin: the next step starts with a list check
};

// With a Verlet skin the sphere and polyhedron paths run in blocks of
// kListCheckEvery steps, blocks starting on multiples of it (counted from the
// simulation's first step).  The step before a block start records the
// largest path since the last re-sort and the largest speed; the gate of the
// block start re-sorts when path_max + look speed_max exceeds half the skin
// (look = 2 kListCheckEvery dt: a particle at rest struck by the fastest one
// reaches at most about twice its speed), and picks the block's mode:
//   fast   (look speed_max <= skin / 4: a fresh list outlasts the block with
//          a factor of two to spare): no check inside the block; every step
//          verifies that no particle has passed half the skin (the bound
//          under which the list holds every contact) and raises
//          kStatusStaleList if one has;
//   exact  (otherwise): a check before every step, re-sorting when a
//          particle has passed half the skin, as without blocks.
// From a forced re-sort (new state, fill wave, removal, new options) to the
// next block start every step ends with a recorded check, so a state that
// starts fast is looked at before its first unchecked step.
constexpr int kListCheckEvery = 8;
// The maxima are spread over kChkSlots words (warp w adds to slot
// w % kChkSlots), so that the atomics of a million particles do not queue on
// one address; the gate reduces the slots with kChkSlots threads.
constexpr int kChkSlots = 128;
constexpr int kChkStride = 32;   // words between slots (one 128-byte line each)
// Returns whether this particle asks for a re-sort before the next step
// (always without a skin); with a skin and check_next, adds its path and
// speed to the maxima instead (one atomic per warp; the gate decides).
__device__ __forceinline__ bool list_needs_rebuild(float skin, const StepLink& link, int exact,
                                                   float path, float speed, StepCtl* ctl,
                                                   uint32_t& st) {
  if (skin <= 0.0f) return true;
  if (link.check_next) {
    const unsigned m = __activemask();
    const uint32_t pm = __reduce_max_sync(m, __float_as_uint(fmaxf(path, 0.0f)));
    const uint32_t vm = __reduce_max_sync(m, __float_as_uint(fmaxf(speed, 0.0f)));
    if ((threadIdx.x & 31) == (__ffs(m) - 1) && ctl->chk) {
      const uint32_t slot =
          ((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % kChkSlots) * kChkStride;
      atomicMax(ctl->chk + slot, pm);
      atomicMax(ctl->chk + kChkSlots * kChkStride + slot, vm);
    }
    return false;
  }
  if (exact) return path > 0.5f * skin;
  if (path > 0.5f * skin) st |= kStatusStaleList;
  return false;
}

struct WallGrid {       // per-cell candidate wall ops (CSR), optional
  const uint32_t* off;  // ncell_tab + 1 entries, or null = test every op
  const uint16_t* ops;
};

// Device copy of the host-side arrays of the reference interface (AoS
// float3 positions/velocities, type, P_ID) and two result words: [0] the
// number of removed particles (P_ID < 0), [1] nonzero when any angular
// velocity is non-zero.
struct HostStage {
  float* pos3;
  float* quat4;   // polyhedra: (w, x, y, z) per particle
  float* vel3;
  float* avel3;
  uint32_t* type;
  int* pid;
  int* flags;
};

// skin > 0: the gate also re-sorts when the maxima recorded by the step
// before it say so, and at a block start picks the block's mode
// (list_needs_rebuild); look = 2 kListCheckEvery dt; vwall = the largest
// surface speed of a moving wall or volume object, counted at a block start
// as a particle speed (a wall can set a resting particle in motion).
void launch_gate(StepCtl* ctl, cudaStream_t st, float skin = 0.0f, float look = 0.0f,
                 int block_start = 0, float vwall = 0.0f);
void launch_gate_graph(StepCtl* ctl, cudaGraphConditionalHandle h0, int* rb, int nrb,
                       cudaStream_t st, float skin = 0.0f, float look = 0.0f);
// Block-start gate of skin > 0 graph stepping: the first node of a block
// graph, followed by a SWITCH node on `hs` whose body it picks on the
// device: 0 keep the list, 1 re-sort then step, 2 exact (a check before
// every step).  The re-sort decision also goes to ctl->gate_r and rb[0]
// (rb[1..nrb) are cleared), the mode to ctl->exact; an exact block's first
// IF takes ctl->gate_r through launch_gate_body.
void launch_gate_switch(StepCtl* ctl, cudaGraphConditionalHandle hs, int* rb, int nrb, float skin,
                        float look, float vwall, cudaStream_t st);
void launch_gate_body(StepCtl* ctl, cudaGraphConditionalHandle h0, cudaStream_t st);
// The gate of plain stepping (launch_gate) as the first node of a one-step
// graph: its decision also sets the IF node `h` of the step's re-sort.
void launch_gate_if(StepCtl* ctl, cudaGraphConditionalHandle h, float skin, float look,
                    int block_start, float vwall, cudaStream_t st);
void launch_hash(const SimParams* dp, const StateBuf& s, const OrderBuf& ob, int n_max,
                 uint32_t* keys, StepCtl* ctl, const int* gate, cudaStream_t st);
// (flat_n, when given, is reset for the contact-list kernel's flat list)
void launch_reorder(const StateBuf& src, const StateBuf& dst, const OrderBuf& ob, int n_max,
                    const uint32_t* sorted_keys, const int32_t* perm, uint32_t* cell_start,
                    uint32_t* cell_end, uint32_t ncell_tab, bool has_lift, int* flat_n,
                    StepCtl* ctl, const int* gate, cudaStream_t st);
void launch_nlist(const SimParams* dp, const StateBuf& s, int n_max, const uint32_t* cell_start,
                  const uint32_t* cell_end, NbrList nl, StepCtl* ctl, const int* gate,
                  cudaStream_t st);
// eb: when not null, the step also writes each particle's energy-tally
// values (particle-particle, volume objects, world objects; FP64) to
// eb[c * n_max + i].  fast: the contracted particle-particle law (ignored
// when eb is given: tallies use the reference's arithmetic).
void launch_step(const SimParams* dp, const WallOp* ops, WallGrid wg, const StateBuf& in_plain,
                 const StateBuf& in_sorted, const StateBuf& out, const OrderBuf& ob, int n_max,
                 NbrList nl, StepCtl* ctl, StepLink link, bool spin_free,
                 const ForceCapture* cap, double* eb, bool fast, cudaStream_t st);
// tally[c] += sum of eb[c * n_max + i] over the current particles, in a fixed
// order; part holds 3 doubles per block of kEnergyBlock particles.
constexpr int kEnergyBlock = 256;
// Self-check of div3_rn against IEEE division on n random triples:
// *bad += the components that differ.
void launch_check_div(long long n, unsigned long long seed, unsigned long long* bad,
                      cudaStream_t st);
void launch_energy_reduce(const double* eb, int n_max, const StepCtl* ctl, double* part,
                          double* tally, cudaStream_t st);
// One step of the mill driver's moves of volume objects: with `turn`, the
// drum's turn of the attached ones (c, s: cosine and sine of the step
// angle, about: the drum axis); then object `translate` (-1: none) moves by
// its velocity times dt.
void launch_move_dobj(SimParams* dp, int turn, float about_x, float about_y, float c, float s,
                      int translate, int n_dobj, cudaStream_t st);
// One step of the turn of the rotating world objects (bit k of rot_mask:
// world object k) on the wall program.
void launch_rotate_wobj(WallOp* ops, int n_ops, uint32_t rot_mask, float about_x, float about_y,
                        float c, float s, cudaStream_t st);
// *out += the particles of the current run whose y exceeds height
// (Silo_Stats, main.cpp:253-280; removed ones parked in range count).
void launch_count_above(const float4* pos, const StepCtl* ctl, int n_max, float height,
                        unsigned int* out, cudaStream_t st);
void launch_kill(const StateBuf& s, const OrderBuf& ob, int n_max, float kill_height,
                 int rotating, float3 max_size, StepCtl* ctl, cudaStream_t st);

// AoS stage -> SoA float4 state (radius from the particle type, type bits in
// vel4.w), P_ID into `pid_dst`, volume-object history reset to -1, and for
// polyhedra the orientation into `ornt_dst` (identity when none is given).
void launch_pack_state(const SimParams* dp, const HostStage& hs, bool has_vel, bool has_avel,
                       const StateBuf& s, int* pid_dst, int* lift_dst, float4* ornt_dst,
                       bool has_ornt, int n, cudaStream_t st);
// SoA float4 state -> AoS stage (the inverse of launch_pack_state; polyhedron
// positions come back relative to the object file's origin).
void launch_unpack_state(const SimParams* dp, const HostStage& hs, const StateBuf& s,
                         const int* pid_src, const float4* ornt_src, int n, cudaStream_t st);

}  // namespace blaze
