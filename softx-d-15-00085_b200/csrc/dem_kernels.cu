// dem_kernels.cu -- the per-step kernels of the sphere DEM path.
//
// Compiled with -fmad=false: every FP32 expression below keeps the operation
// order of the reference source it cites, and with no contraction to FMA the
// results equal the reference's bit for bit.
//
//   k_gate     one thread: latch the rebuild request for this step
//   k_hash     cell key per particle          (BroadPhase.cuh:20-100)
//   [radix sort, radix_sort.cu]               (BroadPhase.cuh:110-117)
//   k_reorder  gather state into sorted order + cell start/end table
//                                             (BroadPhase.cuh:126-325)
//   k_nlist    27-cell neighbour search       (BroadPhase.cuh:335-513)
//   k_step     particle-particle law + volume objects + world objects +
//              symplectic Euler, fused, one thread per particle, gather only
//                                             (DEM_Kernels_Compute.cuh:12-729,
//                                              Collision_Response.cuh,
//                                              Integration.cuh:6-184)
#include "dem_kernels.cuh"
#include "dem_laws.cuh"

namespace blaze {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int3 grid_pos(const SimParams& P, float3 p) {
  int3 g;
  g.x = (int)floorf((p.x - P.origin.x) / P.cell.x);
  g.y = (int)floorf((p.y - P.origin.y) / P.cell.y);
  g.z = (int)floorf((p.z - P.origin.z) / P.cell.z);
  return g;
}
__device__ __forceinline__ uint32_t grid_hash(const SimParams& P, int3 g) {
  return (uint32_t)((g.x + g.z * P.ncells.z) + (g.y * P.ncells.x) * P.ncells.z);
}
__device__ __forceinline__ bool in_grid(const SimParams& P, int3 g) {
  return g.x >= 0 && g.y >= 0 && g.z >= 0 && g.x < P.ncells.x && g.y < P.ncells.y &&
         g.z < P.ncells.z;
}
__device__ __forceinline__ void flag_status(StepCtl* ctl, uint32_t bits) {
  // one atomic per warp
  const unsigned m = __activemask();
  const uint32_t all = __reduce_or_sync(m, bits);
  if (all && (threadIdx.x & 31) == (__ffs(m) - 1)) atomicOr(&ctl->status, all);
}

// --------------------------------------------------------------------- gate
// A list check prepared by the step before (maxima nonzero) re-sorts when a
// particle might pass half the skin before the next check.
// The gate of a step, run by kChkSlots threads (thread 0 decides): the
// re-sort request, and with a skin the maxima recorded by the step before it
// (nonzero only then), which ask for a re-sort when a particle might pass
// half the skin before the next check; at a block start also the block's
// mode (list_needs_rebuild).  Returns the decision in thread 0.
__device__ __forceinline__ int gate_request(StepCtl* ctl, float skin, float look,
                                            int block_start, float vwall) {
  __shared__ uint32_t sp[kChkSlots / 32], sv[kChkSlots / 32];
  const int t = threadIdx.x;
  uint32_t p = 0u, v = 0u;
  if (skin > 0.0f && ctl->chk) {
    uint32_t* cp = ctl->chk + t * kChkStride;
    uint32_t* cv = ctl->chk + (kChkSlots + t) * kChkStride;
    p = *cp;
    v = *cv;
    if (p) *cp = 0u;
    if (v) *cv = 0u;
  }
  p = __reduce_max_sync(0xffffffffu, p);
  v = __reduce_max_sync(0xffffffffu, v);
  if ((t & 31) == 0) {
    sp[t >> 5] = p;
    sv[t >> 5] = v;
  }
  __syncthreads();
  if (t != 0) return 0;
  for (int w = 1; w < kChkSlots / 32; ++w) {
    p = max(p, sp[w]);
    v = max(v, sv[w]);
  }
  int r = ctl->rebuild_req;
  float vm = 0.0f;
  // at a block start the step before recorded the maxima (all zero for a
  // bed at rest), and a moving wall may set a particle in motion within the
  // block: its surface speed counts as a particle speed
  if ((p | v) || (block_start && vwall > 0.0f)) {
    const float pm = __uint_as_float(p);
    vm = fmaxf(__uint_as_float(v), block_start ? vwall : 0.0f);
    if (!(pm + look * vm <= 0.5f * skin)) r = 1;
  }
  if (block_start) {
    ctl->exact = (skin > 0.0f && !(look * vm <= 0.25f * skin)) ? 1 : 0;
    ctl->exact_blocks += ctl->exact;
  }
  return r;
}

__global__ void k_gate(StepCtl* ctl, float skin, float look, int block_start, float vwall) {
  const int r = gate_request(ctl, skin, look, block_start, vwall);
  if (threadIdx.x != 0) return;
  ctl->rebuilt = r;
  ctl->rebuild_req = 0;
}

__global__ void k_gate_switch(StepCtl* ctl, cudaGraphConditionalHandle hs, int* rb, int nrb,
                              float skin, float look, float vwall) {
  const int r = gate_request(ctl, skin, look, 1, vwall);
  if (threadIdx.x != 0) return;
  ctl->rebuild_req = 0;
  ctl->gate_r = r;
  for (int k = 0; k < nrb; ++k) rb[k] = k == 0 ? r : 0;
  cudaGraphSetConditional(hs, ctl->exact ? 2u : (r ? 1u : 0u));
}

__global__ void k_gate_if(StepCtl* ctl, cudaGraphConditionalHandle h, float skin, float look,
                          int block_start, float vwall) {
  const int r = gate_request(ctl, skin, look, block_start, vwall);
  if (threadIdx.x != 0) return;
  ctl->rebuilt = r;
  ctl->rebuild_req = 0;
  cudaGraphSetConditional(h, r ? 1u : 0u);
}

__global__ void k_gate_body(StepCtl* ctl, cudaGraphConditionalHandle h0) {
  cudaGraphSetConditional(h0, ctl->gate_r ? 1u : 0u);
}

// First node of a step graph: latch the request carried over from the last
// launch into the first step's IF condition and clear the per-step
// "re-sorted" flags (an IF body marks its own step).
__global__ void k_gate_graph(StepCtl* ctl, cudaGraphConditionalHandle h0, int* rb, int nrb,
                             float skin, float look) {
  const int r = gate_request(ctl, skin, look, 0, 0.0f);
  if (threadIdx.x != 0) return;
  ctl->rebuild_req = 0;
  for (int k = 0; k < nrb; ++k) rb[k] = 0;
  cudaGraphSetConditional(h0, r ? 1u : 0u);
}

// --------------------------------------------------------------------- hash
// Kernel_SpatialDecomp_CalcPHash (Collision_Detection_BroadPhase.cuh:75-100).
// Removed particles (pid -1) take the largest key so they sort last, as the
// reference's parking position max_size makes them; a live particle outside
// the grid takes the key just below (the reference's table would be indexed
// out of range) and raises kStatusOutOfGrid.
__global__ void __launch_bounds__(kThreads)
k_hash(const SimParams* __restrict__ P, const float4* __restrict__ pos, OrderBuf ob, int n_max,
       uint32_t* __restrict__ keys, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_max) return;
  const int* pid = (ctl->epoch & 1) ? ob.pid[1] : ob.pid[0];
  uint32_t key;
  uint32_t st = 0;
  // removed particles and those a fill has not reached yet stay at the end
  if (pid[i] < 0 || i >= ctl->n_cur) {
    key = P->ncell_tab + 1u;
  } else {
    const float4 p = pos[i];
    const int3 g = grid_pos(*P, xyz(p));
    if (in_grid(*P, g)) {
      key = grid_hash(*P, g);
    } else {
      key = P->ncell_tab;
      st = kStatusOutOfGrid;
    }
  }
  keys[i] = key;
  flag_status(ctl, st);
}

// ------------------------------------------------------------------ reorder
// Kernel_SortArrays + Kernel_SpatialDecomp_ReorderPDA + Kernel_SpatialDecomp_BinData
// (BroadPhase.cuh:126-325), as one gather into the spare buffer.
__global__ void __launch_bounds__(kThreads)
k_reorder(StateBuf src, StateBuf dst, OrderBuf ob, int n_max,
          const uint32_t* __restrict__ keys, const int32_t* __restrict__ perm,
          uint32_t* __restrict__ cstart, uint32_t* __restrict__ cend, uint32_t ncell_tab,
          int has_lift, int* flat_n, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = ctl->epoch & 1;
  if (i == 0) {
    // the particles removed since the last re-sort are now at the end
    ctl->n_cur -= ctl->pending_dead;
    ctl->pending_dead = 0;
    if (flat_n) *flat_n = 0;  // the contact-list kernel lists the slots anew
  }
  if (i >= n_max) return;
  const int j = perm[i];
  dst.pos[i] = src.pos[j];
  dst.vel[i] = src.vel[j];
  float4 w = src.angv[j];
  w.w = 0.0f;
  dst.angv[i] = w;
  const int* pid_src = e ? ob.pid[1] : ob.pid[0];
  int* pid_dst = e ? ob.pid[0] : ob.pid[1];
  pid_dst[i] = pid_src[j];
  if (has_lift) {
    const int* l_src = e ? ob.lift[1] : ob.lift[0];
    int* l_dst = e ? ob.lift[0] : ob.lift[1];
    l_dst[i] = l_src[j];
  }
  if (ob.ornt[0]) {
    const float4* q_src = e ? ob.ornt[1] : ob.ornt[0];
    float4* q_dst = e ? ob.ornt[0] : ob.ornt[1];
    q_dst[i] = q_src[j];
  }
  const uint32_t k = keys[i];
  if (k < ncell_tab) {
    if (i == 0 || keys[i - 1] != k) cstart[k] = (uint32_t)i;
    if (i == n_max - 1 || keys[i + 1] != k) cend[k] = (uint32_t)i + 1u;
  }
}

// -------------------------------------------------------------------- nlist
// Kernel_BroadCollisionDetection_NonSymmetry (BroadPhase.cuh:402-513) with
// CollisionDetection_Filter_SphereNNCell (BroadPhase.cuh:335-392): the
// clamped 3x3x3 block scanned in y, z, x order, j ascending inside a cell,
// pairs kept when |xi - xj| - (ri + rj) < 0 (skin 0: the reference's
// contacts-only list, bit for bit), or with a skin every pair with
// |xi - xj| < ri + rj + skin (up to a relative 2^-20 more).  Slots beyond the capacity are dropped and flagged
// (the reference writes past its 32-slot row).
__global__ void __launch_bounds__(kThreads)
k_nlist(const SimParams* __restrict__ P, const float4* __restrict__ pos, int n_max,
        const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, NbrList nl,
        StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ctl->epoch += 1;
  const int n = ctl->n_cur;
  if (i >= n) return;
  const float4 pa4 = pos[i];
  const float3 pa = xyz(pa4);
  const float ra = pa4.w;
  const float skin = P->skin;
  const int3 g = grid_pos(*P, pa);
  uint32_t cnt = 0;
  uint32_t st = 0;
  // a pair within the skin is at most 2 max(ra, rb) + skin apart: the
  // larger sphere of every pair checks that this fits in one cell edge
  if (skin > 0.0f && 2.0f * ra + skin > fminf(P->cell.x, fminf(P->cell.y, P->cell.z)))
    st |= kStatusCellTooSmall;
  if (in_grid(*P, g)) {
    const int xs = g.x == 0 ? 0 : -1, xe = g.x == P->ncells.x - 1 ? 0 : 1;
    const int ys = g.y == 0 ? 0 : -1, ye = g.y == P->ncells.y - 1 ? 0 : 1;
    const int zs = g.z == 0 ? 0 : -1, ze = g.z == P->ncells.z - 1 ? 0 : 1;
    for (int y = ys; y <= ye; ++y)
      for (int z = zs; z <= ze; ++z)
        for (int x = xs; x <= xe; ++x) {
          const uint32_t h = grid_hash(*P, make_int3(g.x + x, g.y + y, g.z + z));
          const uint32_t s = __ldg(cstart + h);
          if (s == 0xffffffffu) continue;
          const uint32_t e = __ldg(cend + h);
          for (uint32_t j = s; j < e; ++j) {
            if ((int)j == i) continue;
            const float4 pb = __ldg(pos + j);
            const float3 rel = pa - xyz(pb);
            const float sr = ra + pb.w;
            // skin 0: the reference's test, decided without the square root
            // where that is exact (touches); with a skin the list need only
            // hold every pair within it, so a bound a hair wider serves
            bool keep;
            if (skin > 0.0f) {
              const float reach = sr + skin;
              keep = dot3(rel, rel) < (reach * reach) * (1.0f + 0x1p-20f);
            } else {
              keep = touches(rel, sr);
            }
            if (keep) {
              if (cnt < (uint32_t)nl.cap) nl.idx[(size_t)cnt * nl.stride + i] = j;
              else st |= kStatusListOverflow;
              ++cnt;
            }
          }
        }
  }
  const uint32_t kept = cnt < (uint32_t)nl.cap ? cnt : (uint32_t)nl.cap;
  nl.cnt[i] = kept;
  if (nl.flat) {
    // append this particle's slots to the flat list: one atomic per warp;
    // the lanes still here (i < n) are a prefix of the warp
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31;
    uint32_t x = kept;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(m, x, d);
      if (lane >= d) x += y;
    }
    const int last = 31 - __clz((int)m);
    uint32_t base = 0;
    if (lane == last) base = (uint32_t)atomicAdd(nl.flat_n, (int)x);
    base = __shfl_sync(m, base, last) + (x - kept);
    for (uint32_t k = 0; k < kept; ++k) nl.flat[base + k] = k * (uint32_t)nl.stride + (uint32_t)i;
  }
  flag_status(ctl, st);
}


// WorldObject_InteractionParticle for spheres (DEM_Kernels_Compute.cuh:254-610):
// one op per face / plane / cylinder / cap in world-object order.
// es: when not null, the contact's energy-tally value is added to *es.
template <bool kSpin>
__device__ __forceinline__ void apply_wall_op(const SimParams& P, const WallOp& op, float3 p,
                                              float r, float3 v, float3 w, const TypeParams& T,
                                              float3& fw, float3& tw, double* es = nullptr) {
  float e = 0.0f;
  float* ep = es ? &e : nullptr;
  if (op.kind == kOpFace || op.kind == kOpPlane) {
    // Collision_Detection_Sphere_Surface / _Plane, Collision_Detection_Spheres.cuh:6-100
    const float3 pt = p - r * op.n;
    float dis = dot3(op.n, pt - op.c);
    if (!(dis < 0.000000f && dis > -r)) return;
    dis = fabsf(dis);
    if (op.kind == kOpFace) {
      const float3 q = pt + op.n * dis;
      if (!point_on_polygon(op.nv, op.v, q, op.area, op.tol)) return;
    }
    Forces F;
    if (P.rotating_wobj && P.cyl_rot)
      F = law_moving_surface<kSpin>(P, op.n, dis, pt - p, w, T, v, drum_velocity(P, pt), ep);
    else
      F = law_static_surface(P, v, op.n, dis, pt - p, w, T, ep);
    fw = fw + F.trans;
    if (P.rotation) tw = tw + F.torque;
    if (es) *es += (double)e;
  } else if (op.kind == kOpCylinder) {
    // Collision_Detection_Sphere_Cylinder, Collision_Detection_Spheres.cuh:234-265
    const float3 pv = vmul(p, op.axis) - op.cbot;
    const float pd = len3(pv) + r;
    if (!(pd > op.radius)) return;
    float3 nrm = f3(-pv.x, -pv.y, -pv.z);
    nrm = nrm * (1.0f / len3(nrm));
    const float3 cp = p - nrm * r;
    const float dis = fabsf(pd - op.radius);
    Forces F;
    if (P.cyl_rot)
      F = law_moving_surface<kSpin>(P, nrm, dis, cp - p, w, T, v, drum_velocity(P, cp), ep);
    else
      F = law_static_surface(P, v, nrm, dis, cp - p, w, T, ep);
    fw = F.trans;
    if (P.rotation) tw = tw + F.torque;
    if (es) *es += (double)e;
  } else {
    // end plates: Collision_Detection_Sphere_Plane + Collision_Response_EndPlate_Particle
    const float3 pt = p - r * op.n;
    float dis = dot3(op.n, pt - op.c);
    if (!(dis < 0.000000f && dis > -r)) return;
    dis = fabsf(dis);
    fw = law_end_plate(v, op.n, dis, T);
  }
}

// Collision_Detection_Sphere_DObject, Collision_Detection_Spheres.cuh:108-225
struct DobjHit { bool hit; int type; float dis; float3 n, cp; };
__device__ __forceinline__ DobjHit sphere_dobject(const DobjDev& D, float3 p, float r,
                                                  int hist_type) {
  DobjHit c;
  c.hit = false;
  c.type = 0;
  if (hist_type != 2) {
    for (int j = 0; j < D.num_faces; ++j) {
      const Surface& s = D.faces[j];
      const float3 pt = p - r * s.normal;
      float dis = dot3(s.normal, pt - s.centroid);
      if (dis < 0.000000f && dis > -r * 0.50f) {
        dis = fabsf(dis);
        const float3 q = pt + s.normal * dis;
        const int nv = s.num_vertex < 8 ? s.num_vertex : 8;
        if (point_on_indexed_polygon(nv, D.vert, s.vertex_Order, q, s.area, s.Tol)) {
          c.hit = true; c.type = 1; c.dis = dis; c.n = s.normal; c.cp = pt;
          return c;
        }
      }
    }
  }
  for (int e = 0; e < D.num_edges; ++e) {
    const float3 p0 = D.vert[D.edge0[e]];
    const float3 dir = D.vert[D.edge1[e]] - p0;
    const float3 edir = dir / len3(dir);
    const float dvec = dot3(edir, p - p0);
    if (dvec > 0) {
      const float3 p2 = p0 + dvec * edir;
      const float3 d2 = p - p2;
      const float d = len3(d2);
      if (d < r) {
        const float dis = fabsf(d - r);
        if (dis < r) {
          c.n = d2 * (1.0f / len3(d2));
          c.cp = f3(0.0f, 0.0f, 0.0f);
          c.type = 2; c.hit = true; c.dis = dis;
          return c;
        }
      }
    }
  }
  return c;
}

// ---------------------------------------------------------------------- step
#ifndef BLAZE_STEP_MIN_BLOCKS
#define BLAZE_STEP_MIN_BLOCKS 4
#endif
// candidate slots tested per batch of independent loads in the contact pass
// (settled 1M silo, contracted law, ms a step: 4 0.123, 5 0.122, 6 0.121,
// 7 0.120, 8 0.125, 12 0.142, 16 0.161; wider batches spill)
constexpr int kMaskBatch = 7;


// kEnergy: also the energy tallies of the step's contacts, per particle in
// contact order (particle-particle, volume objects, world objects), into
// eb[c * n_max + i] in FP64.
// kFast: the particle-particle law in contracted form (law_pp_fast) and the
// contact normal from an approximate reciprocal; contact tests, walls, volume
// objects and the integrator are unchanged.  Not with kEnergy.
template <bool kCapture, bool kSpin, bool kEnergy, bool kFast>
__global__ void __launch_bounds__(kThreads, BLAZE_STEP_MIN_BLOCKS)
k_step(const SimParams* __restrict__ Pg, const WallOp* __restrict__ ops, WallGrid wg,
       StateBuf in_plain, StateBuf in_sorted, StateBuf out, OrderBuf ob, int n_max,
       NbrList nl, StepCtl* ctl, StepLink link, ForceCapture cap, double* eb) {
  __shared__ TypeParams sT[kMaxTypes];
  {
    const int words = (int)(sizeof(TypeParams) * kMaxTypes / 4);
    const int* src = reinterpret_cast<const int*>(Pg->types);
    int* dst = reinterpret_cast<int*>(sT);
    for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
  }
  __syncthreads();
  const SimParams& P = *Pg;
  const bool rebuilt = *link.rebuilt != 0;
  const StateBuf in = rebuilt ? in_sorted : in_plain;
  const int n = ctl->n_cur;
  const int exact = ctl->exact;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_max) return;
  if (i >= n) {  // removed particles keep their parked state
    out.pos[i] = in.pos[i];
    out.vel[i] = in.vel[i];
    out.angv[i] = in.angv[i];
    return;
  }
  const float4 pa4 = in.pos[i], va4 = in.vel[i], wa4 = in.angv[i];
  const float3 pa = xyz(pa4), va = xyz(va4), wa = xyz(wa4);
  const int ta = __float_as_int(va4.w);
  const TypeParams& TA = sT[ta & (kMaxTypes - 1)];
  const float ma = TA.mass, ra = pa4.w;
  uint32_t st = (ta < 0 || ta >= P.n_types) ? kStatusTypeRange : 0u;

  // particle-particle (Kernel_ParticleInteraction_Spheres_NonSymmetry)
  float3 f = P.gravity * ma;
  float3 fl = f3(0.0f, 0.0f, 0.0f);
  double e_pp = 0.0, e_lift = 0.0, e_surf = 0.0;
  float ec = 0.0f;
  // contacts first (the slots whose spheres overlap), candidates in batches:
  // all index loads of a batch, then all position gathers, then the tests,
  // so a batch costs one round trip per level
  const int cnt = (int)nl.cnt[i];
  const uint32_t* __restrict__ li = nl.idx + i;
  uint32_t cm = 0;
  for (int k0 = 0; k0 < cnt; k0 += kMaskBatch) {
    uint32_t jj[kMaskBatch];
#pragma unroll
    for (int u = 0; u < kMaskBatch; ++u)
      jj[u] = k0 + u < cnt ? __ldg(li + (size_t)(k0 + u) * nl.stride) : 0u;
    float4 pb[kMaskBatch];
#pragma unroll
    for (int u = 0; u < kMaskBatch; ++u)
      pb[u] = k0 + u < cnt ? __ldg(in.pos + jj[u]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int u = 0; u < kMaskBatch; ++u) {
      if (k0 + u < cnt && touches(pa - xyz(pb[u]), ra + pb[u].w)) cm |= 1u << (k0 + u);
    }
  }
  // the contacts in slot order, the next contact's gathers issued before
  // this contact's law
  float4 pn4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), vn4 = pn4, wn4 = pn4;
  bool more = cm != 0u;
  if (more) {
    const int j = (int)li[(size_t)(__ffs(cm) - 1) * nl.stride];
    cm &= cm - 1u;
    pn4 = __ldg(in.pos + j);
    vn4 = __ldg(in.vel + j);
    if (kSpin) wn4 = __ldg(in.angv + j);
  }
  while (more) {
    const float4 pb4 = pn4, vb4 = vn4, wb4 = wn4;
    more = cm != 0u;
    if (more) {
      const int j = (int)li[(size_t)(__ffs(cm) - 1) * nl.stride];
      cm &= cm - 1u;
      pn4 = __ldg(in.pos + j);
      vn4 = __ldg(in.vel + j);
      if (kSpin) wn4 = __ldg(in.angv + j);
    }
    const float3 rel = pa - xyz(pb4);
    const float dist = len3(rel);
    const int tb = __float_as_int(vb4.w);
    const float3 vb = xyz(vb4);
    const float dis = fabsf(dist - (ra + pb4.w)) + 0.000010f;
    const PP_Parms& pp = TA.pp[tb < kMaxPP ? tb : 0];
    Forces F;
    if constexpr (kFast) {
      const float3 nrm = rel * __fdividef(1.0f, dist);
      F = law_pp_fast<kSpin>(P, va - vb, nrm, dis, nrm * (-ra), nrm * pb4.w, wa, xyz(wb4), pp, va,
                             vb, (P.tan_k * pp.Fric_kinetic) * (ma + sT[tb & (kMaxTypes - 1)].mass));
    } else {
      const float3 nrm = div3_rn(rel, dist);   // = rel / dist, three correctly rounded quotients
      F = law_pp<kSpin>(P, va - vb, nrm, dis, (-1.0f * nrm) * ra, nrm * pb4.w, wa, xyz(wb4), pp,
                        va, vb, ma, sT[tb & (kMaxTypes - 1)].mass, kEnergy ? &ec : nullptr);
    }
    f = f + F.trans;
    fl = fl + F.torque;
    if (kEnergy) e_pp += (double)ec;
  }
  const float3 f_pp = f;
  const float3 t_pp = P.rotation ? fl : f3(0.0f, 0.0f, 0.0f);

  // volume objects (VolumeObject_InteractionParticle, DEM_Kernels_Compute.cuh:12-246)
  float3 f_l = f3(0.0f, 0.0f, 0.0f), t_l = f3(0.0f, 0.0f, 0.0f);
  if (P.n_dobj > 0) {
    int* lift = (ctl->epoch & 1) ? ob.lift[1] : ob.lift[0];
    const int hist = lift[i];
    int colltype = 0;
    bool outer = P.dobj[0].translating || !P.is_mill || P.rotating_wobj;
    if (!outer) outer = len3(f3(pa.x, pa.y, 0.0f) - P.cent) > (P.dobj_cyl_bound_r - 2.0f * TA.radius);
    if (outer) {
      for (int d = 0; d < P.n_dobj; ++d) {
        const DobjDev& D = P.dobj[d];
        const float3 bv = vmul(pa - D.com, D.axis);
        if (!(len3(bv) < (D.bound_r + TA.radius))) continue;
        DobjHit c = sphere_dobject(D, pa, TA.radius, hist);
        colltype = c.type;
        if (c.hit) {
          if (c.type == 2) c.cp = pa;
          float3 vobj = f3(0.0f, 0.0f, 0.0f);
          if (D.attached) vobj = drum_velocity(P, c.cp);
          else if (D.translating) vobj = D.velocity;
          const Forces F = law_volume<kSpin>(P, c.n, c.dis, c.cp - pa, wa, TA, va, vobj,
                                             kEnergy ? &ec : nullptr);
          f_l = f_l + F.trans;
          if (P.rotation) t_l = t_l + F.torque;
          if (kEnergy) e_lift += (double)ec;
          break;
        }
      }
    }
    lift[i] = colltype;
  }

  // world objects
  float3 f_w = f3(0.0f, 0.0f, 0.0f), t_w = f3(0.0f, 0.0f, 0.0f);
  if (wg.off != nullptr) {
    const int3 g = grid_pos(P, pa);
    if (in_grid(P, g)) {
      const uint32_t h = grid_hash(P, g);
      const uint32_t o0 = __ldg(wg.off + h), o1 = __ldg(wg.off + h + 1);
      for (uint32_t q = o0; q < o1; ++q)
        apply_wall_op<kSpin>(P, ops[__ldg(wg.ops + q)], pa, ra, va, wa, TA, f_w, t_w,
                             kEnergy ? &e_surf : nullptr);
    } else {
      for (int q = 0; q < P.n_ops; ++q)
        apply_wall_op<kSpin>(P, ops[q], pa, ra, va, wa, TA, f_w, t_w, kEnergy ? &e_surf : nullptr);
    }
  } else {
    for (int q = 0; q < P.n_ops; ++q)
      apply_wall_op<kSpin>(P, ops[q], pa, ra, va, wa, TA, f_w, t_w, kEnergy ? &e_surf : nullptr);
  }
  if (kEnergy) {
    eb[i] = e_pp;
    eb[(size_t)n_max + i] = e_lift;
    eb[2 * (size_t)n_max + i] = e_surf;
  }
  if (!P.rotation) t_w = f3(0.0f, 0.0f, 0.0f);

  // Integrate_Euler_NonSymmetry (Integration.cuh:6-184), spheres
  float3 acc = f_w + f_pp;
  if (P.n_dobj > 0) acc = acc + f_l;
  acc = acc * (1.0f / ma);
  float3 v = va + acc * P.dt;
  const float3 p = pa + v * P.dt;
  if (P.mode2d) v.z = 0.0f;
  float3 tl = t_pp + t_w;
  if (P.n_dobj > 0) tl = tl + t_l;
  float3 w = wa;
  if (P.rotation) {
    if (dot3(tl, tl) > 0.0f) {
      const float3 aa = TA.iinv * tl;
      w = w + aa * P.dt;
      w = w - w * P.roll_res;
    }
    if (P.mode2d) { w.x = 0.0f; w.y = 0.0f; }
  }
  float path = wa4.w;
  if (P.skin > 0.0f) path = path + len3(v) * P.dt;
  out.pos[i] = make_float4(p.x, p.y, p.z, ra);
  out.vel[i] = make_float4(v.x, v.y, v.z, va4.w);
  out.angv[i] = make_float4(w.x, w.y, w.z, path);
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) st |= kStatusNonFinite;

  // Verlet-list validity (list_needs_rebuild); with no skin the contact list
  // is rebuilt every step (reference).
  {
    const unsigned m = __activemask();
    const bool need = list_needs_rebuild(P.skin, link, exact, path, len3(v), ctl, st);
    const unsigned b = __ballot_sync(m, need);
    if (b && (threadIdx.x & 31) == (__ffs(m) - 1)) {
      if (link.has_next_h) cudaGraphSetConditional(link.next_h, 1u);
      else atomicExch(&ctl->rebuild_req, 1);
    }
  }
  flag_status(ctl, st);

  if (kCapture) {
    const float3 vals[6] = {f_pp, t_pp, f_w, t_w, f_l, t_l};
    float* dsts[6] = {cap.f_pp, cap.t_pp, cap.f_w, cap.t_w, cap.f_l, cap.t_l};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      dsts[q][3 * i] = vals[q].x;
      dsts[q][3 * i + 1] = vals[q].y;
      dsts[q][3 * i + 2] = vals[q].z;
    }
  }
}

// ------------------------------------------------------------ energy tallies
// Sum of eb over the current particles, category by category, added to
// tally[3]: per block a fixed tree over its particles, then one block over
// the block sums in block order, so the result does not depend on timing.
__global__ void __launch_bounds__(kEnergyBlock)
k_energy_partial(const double* __restrict__ eb, int n_max, const StepCtl* ctl,
                 double* __restrict__ part) {
  __shared__ double sh[3][kEnergyBlock];
  const int n = ctl->n_cur;
  const int i = blockIdx.x * kEnergyBlock + threadIdx.x;
#pragma unroll
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = i < n ? eb[(size_t)c * n_max + i] : 0.0;
  __syncthreads();
  for (int w = kEnergyBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[3 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(kEnergyBlock)
k_energy_final(const double* __restrict__ part, int nb, double* tally) {
  __shared__ double sh[3][kEnergyBlock];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += kEnergyBlock)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += part[3 * b + c];
#pragma unroll
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = kEnergyBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) tally[threadIdx.x] += sh[threadIdx.x][0];
}

// ------------------------------------------------------- kinematic world
// The mill driver's per-step moves of volume and world objects
// (Processing_Mills.h), on the device, in the host functions' FP32 operation
// order; c and s are the host's cosf / sinf of the step angle.

// x' = c x + s y, y' = -s x + c y about `about` (z unchanged).
__device__ __forceinline__ float3 turn_about(float3 v, float3 about, float c, float s) {
  const float3 p = v - about;
  v.x = c * p.x + s * p.y;
  v.y = (-s) * p.x + c * p.y;
  return v + about;
}

// A volume object's faces from its vertices: centroid, normal cross(V2, V1)
// normalised, area of the quad (Processing_Mills.h:27-58).
__device__ void dobj_faces(DobjDev& D) {
  for (int j = 0; j < D.num_faces; ++j) {
    Surface& F = D.faces[j];
    float3 sum = f3(0.0f, 0.0f, 0.0f);
    for (int q = 0; q < F.num_vertex && q < 8; ++q) sum = sum + D.vert[F.vertex_Order[q] & 7];
    F.centroid = (1.0f / (float)F.num_vertex) * sum;
    const int* o = F.vertex_Order;
    const float3 v1 = D.vert[o[1] & 7] - D.vert[o[0] & 7];
    const float3 v2 = D.vert[o[2] & 7] - D.vert[o[1] & 7];
    const float3 v3 = D.vert[o[3] & 7] - D.vert[o[2] & 7];
    const float3 v4 = D.vert[o[0] & 7] - D.vert[o[3] & 7];
    const float3 nrm = cross3(v2, v1);
    F.normal = nrm / len3(nrm);
    F.area = 0.500000f * len3(nrm) + 0.500000f * len3(cross3(v3, v4));
  }
}

// Rotate_VolObject_Inc (Processing_Mills.h:4-75): every volume object
// attached to the drum turns about `about` (x, y; z = 0): vertices and
// centre of mass, then its faces.  Translate_VolObject
// (Processing_Mills.h:336-396), after the turn: object `tr` (or none, -1)
// moves by its velocity times dt.
__global__ void k_move_dobj(SimParams* P, int turn, float about_x, float about_y, float c,
                            float s, int tr) {
  const int d = threadIdx.x;
  if (d >= P->n_dobj) return;
  DobjDev& D = P->dobj[d];
  if (turn && D.attached) {
    const float3 about = f3(about_x, about_y, 0.0f);
    for (int k = 0; k < D.num_vertex; ++k) D.vert[k] = turn_about(D.vert[k], about, c, s);
    dobj_faces(D);
    D.com = turn_about(D.com, about, c, s);
  }
  if (d == tr) {
    const float3 disp = D.velocity * P->dt;
    for (int k = 0; k < D.num_vertex; ++k) D.vert[k] = D.vert[k] + disp;
    dobj_faces(D);
    D.com = D.com + disp;
  }
}

// Rotate_WObject_inc (Processing_Mills.h:257-334) on the wall program: each
// face (or plane) of a rotating world object (bit `wobj` of rot_mask) has
// its vertices turned, then centroid, normal cross(V2, V1) normalised and
// area (quad: both triangles; triangle: one); every face copy of a shared
// vertex turns the same number to the same result.
__global__ void k_rotate_wobj(WallOp* ops, int n_ops, uint32_t rot_mask, float about_x,
                              float about_y, float c, float s) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_ops) return;
  WallOp& op = ops[q];
  if (op.kind != kOpFace && op.kind != kOpPlane) return;
  if (op.wobj < 0 || op.wobj > 31 || !((rot_mask >> op.wobj) & 1u)) return;
  const float3 about = f3(about_x, about_y, 0.0f);
  for (int k = 0; k < op.nv; ++k) op.v[k] = turn_about(op.v[k], about, c, s);
  float3 sum = f3(0.0f, 0.0f, 0.0f);
  for (int k = 0; k < op.nv; ++k) sum = sum + op.v[k];
  op.c = (1.0f / (float)op.nv) * sum;
  const float3 v1 = op.v[1] - op.v[0];
  const float3 v2 = op.v[2] - op.v[1];
  const float3 nrm = cross3(v2, v1);
  op.n = nrm / len3(nrm);
  if (op.nv > 3) {
    const float3 v3 = op.v[3] - op.v[2];
    const float3 v4 = op.v[0] - op.v[3];
    op.area = 0.500000f * len3(nrm) + 0.500000f * len3(cross3(v3, v4));
  } else {
    op.area = 0.500000f * len3(nrm);
  }
  op.kind = op.area == -1.0f ? kOpPlane : kOpFace;
}

// --------------------------------------------------------- division check
// div3_rn against three IEEE divisions on n pseudo-random triples (a
// SplitMix64 stream per index: numerators over 1e-25..1e25 and both signs,
// denominators over 1e-18..1e18, one in 64 numerators zero or a signed
// power of two), counting the components that differ in any bit.
__device__ __forceinline__ unsigned long long splitmix(unsigned long long& x) {
  unsigned long long z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ float log_uniform(unsigned long long u, float lo_exp, float hi_exp) {
  const float t = (float)(u >> 40) * (1.0f / 16777216.0f);
  return exp10f(lo_exp + t * (hi_exp - lo_exp));
}
__global__ void k_check_div(long long n, unsigned long long seed, unsigned long long* bad) {
  unsigned long long local = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long x = seed ^ (unsigned long long)i * 0xD1B54A32D192ED03ull;
    float a[3];
    for (int c = 0; c < 3; ++c) {
      const unsigned long long u = splitmix(x);
      float v = log_uniform(u, -25.0f, 25.0f);
      if ((u & 63ull) == 0) v = 0.0f;
      else if ((u & 63ull) == 1) v = ldexpf(1.0f, (int)((u >> 8) % 120) - 60);
      a[c] = (u >> 7) & 1ull ? -v : v;
    }
    const float b = log_uniform(splitmix(x), -18.0f, 18.0f);
    const float3 q = div3_rn(f3(a[0], a[1], a[2]), b);
    const float r[3] = {q.x, q.y, q.z};
    for (int c = 0; c < 3; ++c)
      if (__float_as_uint(r[c]) != __float_as_uint(__fdiv_rn(a[c], b))) ++local;
  }
  if (local) atomicAdd(bad, local);
}

// ---------------------------------------------------------------------- kill
// Remove_Silo_Discharged_Particles / Remove_PL_Discharged_Particles
// (GPU_Memory_Transfer.cuh:646-682): park at max_size, pid -1, count.  The
// count is per check (the reference's Kill_count is never reset).
__global__ void k_kill(StateBuf s, OrderBuf ob, int n_max, float kill_height, int rotating,
                       float3 max_size, StepCtl* ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = ctl->n_cur;
  if (i >= n || i >= n_max) return;
  int* pid = (ctl->epoch & 1) ? ob.pid[1] : ob.pid[0];
  if (pid[i] == -1) return;
  const float4 p = s.pos[i];
  bool kill;
  if (rotating)
    kill = p.z <= 41.0f || p.z >= 300 || p.y <= 50.0f || p.y >= 1500.0f || p.x <= 50.0f ||
           p.x >= 1500.0f;
  else
    kill = p.y < kill_height;
  if (kill) {
    s.pos[i] = make_float4(max_size.x, max_size.y, max_size.z, p.w);
    pid[i] = -1;
    atomicAdd(&ctl->pending_dead, 1);
    atomicAdd(&ctl->killed_total, 1);
    ctl->rebuild_req = 1;
  }
}

// Silo_Stats (main.cpp:253-280): how many particles of the current run
// (memory positions [0, n_cur)) lie above `height`.  Particles removed since
// the last re-sort are still in that range at the parking position, as the
// reference counts them.  Integer sums: the count does not depend on order.
__global__ void __launch_bounds__(kThreads)
k_count_above(const float4* __restrict__ pos, const StepCtl* ctl, int n_max, float height,
              unsigned int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = min(ctl->n_cur, n_max);
  const unsigned int above = (i < n && pos[i].y > height) ? 1u : 0u;
  const unsigned int w = __reduce_add_sync(0xffffffffu, above);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(out, w);
}

// ------------------------------------------------------------ state staging
// Set_PSystem_State / Get_SystemState (GPU_Memory_Transfer.cuh:377-418,
// 486-520) as one pass each over the staged host arrays.
__global__ void __launch_bounds__(kThreads)
k_pack_state(const SimParams* __restrict__ P, HostStage hs, int has_vel, int has_avel, StateBuf s,
             int* __restrict__ pid_dst, int* __restrict__ lift_dst, float4* __restrict__ ornt_dst,
             int has_ornt, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t t = hs.type[i];
  const float r = t < (uint32_t)P->n_types ? P->types[t].radius : 0.0f;
  const float tb = __int_as_float((int)t);
  s.pos[i] = make_float4(hs.pos3[3 * i], hs.pos3[3 * i + 1], hs.pos3[3 * i + 2], r);
  s.vel[i] = has_vel ? make_float4(hs.vel3[3 * i], hs.vel3[3 * i + 1], hs.vel3[3 * i + 2], tb)
                     : make_float4(0.0f, 0.0f, 0.0f, tb);
  const float4 w = has_avel
                       ? make_float4(hs.avel3[3 * i], hs.avel3[3 * i + 1], hs.avel3[3 * i + 2], 0.0f)
                       : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.angv[i] = w;
  const int id = hs.pid[i];
  pid_dst[i] = id;
  if (lift_dst) lift_dst[i] = -1;
  // Set_PSystem_State (GPU_Memory_Transfer.cuh:400-440): polyhedra take the
  // caller's orientation, positions as given (the centre of mass)
  if (ornt_dst)
    ornt_dst[i] = has_ornt ? make_float4(hs.quat4[4 * i], hs.quat4[4 * i + 1], hs.quat4[4 * i + 2],
                                         hs.quat4[4 * i + 3])
                           : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
  const unsigned m = __activemask();
  const int dead = __popc(__ballot_sync(m, id < 0));
  const bool spin = __any_sync(m, w.x != 0.0f || w.y != 0.0f || w.z != 0.0f);
  if ((threadIdx.x & 31) == (__ffs(m) - 1)) {
    if (dead) atomicAdd(&hs.flags[0], dead);
    if (spin) atomicOr(&hs.flags[1], 1);
  }
}

__global__ void __launch_bounds__(kThreads)
k_unpack_state(const SimParams* __restrict__ P, HostStage hs, StateBuf s,
               const int* __restrict__ pid_src, const float4* __restrict__ ornt_src, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = s.pos[i], v = s.vel[i], w = s.angv[i];
  if (ornt_src) {
    // Get_SystemState (GPU_Memory_Transfer.cuh:486-520): a polyhedron's
    // position is returned relative to its object file's origin (pos - COM)
    const int t = __float_as_int(v.w);
    const float3 c = P->types[t & (kMaxTypes - 1)].com;
    hs.pos3[3 * i] = p.x - c.x; hs.pos3[3 * i + 1] = p.y - c.y; hs.pos3[3 * i + 2] = p.z - c.z;
    const float4 q = ornt_src[i];
    hs.quat4[4 * i] = q.x; hs.quat4[4 * i + 1] = q.y; hs.quat4[4 * i + 2] = q.z;
    hs.quat4[4 * i + 3] = q.w;
  } else {
    hs.pos3[3 * i] = p.x; hs.pos3[3 * i + 1] = p.y; hs.pos3[3 * i + 2] = p.z;
  }
  hs.vel3[3 * i] = v.x; hs.vel3[3 * i + 1] = v.y; hs.vel3[3 * i + 2] = v.z;
  hs.avel3[3 * i] = w.x; hs.avel3[3 * i + 1] = w.y; hs.avel3[3 * i + 2] = w.z;
  hs.type[i] = (uint32_t)__float_as_int(v.w);
  hs.pid[i] = pid_src[i];
}

inline int blocks(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

void launch_gate(StepCtl* ctl, cudaStream_t st, float skin, float look, int block_start,
                 float vwall) {
  k_gate<<<1, kChkSlots, 0, st>>>(ctl, skin, look, block_start, vwall);
}

void launch_gate_switch(StepCtl* ctl, cudaGraphConditionalHandle hs, int* rb, int nrb, float skin,
                        float look, float vwall, cudaStream_t st) {
  k_gate_switch<<<1, kChkSlots, 0, st>>>(ctl, hs, rb, nrb, skin, look, vwall);
}

void launch_gate_if(StepCtl* ctl, cudaGraphConditionalHandle h, float skin, float look,
                    int block_start, float vwall, cudaStream_t st) {
  k_gate_if<<<1, kChkSlots, 0, st>>>(ctl, h, skin, look, block_start, vwall);
}

void launch_gate_body(StepCtl* ctl, cudaGraphConditionalHandle h0, cudaStream_t st) {
  k_gate_body<<<1, 1, 0, st>>>(ctl, h0);
}

void launch_gate_graph(StepCtl* ctl, cudaGraphConditionalHandle h0, int* rb, int nrb,
                       cudaStream_t st, float skin, float look) {
  k_gate_graph<<<1, kChkSlots, 0, st>>>(ctl, h0, rb, nrb, skin, look);
}

void launch_hash(const SimParams* dp, const StateBuf& s, const OrderBuf& ob, int n_max,
                 uint32_t* keys, StepCtl* ctl, const int* gate, cudaStream_t st) {
  k_hash<<<blocks(n_max), kThreads, 0, st>>>(dp, s.pos, ob, n_max, keys, ctl, gate);
}

void launch_reorder(const StateBuf& src, const StateBuf& dst, const OrderBuf& ob, int n_max,
                    const uint32_t* sorted_keys, const int32_t* perm, uint32_t* cell_start,
                    uint32_t* cell_end, uint32_t ncell_tab, bool has_lift, int* flat_n,
                    StepCtl* ctl, const int* gate, cudaStream_t st) {
  k_reorder<<<blocks(n_max), kThreads, 0, st>>>(src, dst, ob, n_max, sorted_keys, perm, cell_start,
                                                cell_end, ncell_tab, has_lift ? 1 : 0, flat_n,
                                                ctl, gate);
}

void launch_nlist(const SimParams* dp, const StateBuf& s, int n_max, const uint32_t* cell_start,
                  const uint32_t* cell_end, NbrList nl, StepCtl* ctl, const int* gate,
                  cudaStream_t st) {
  k_nlist<<<blocks(n_max), kThreads, 0, st>>>(dp, s.pos, n_max, cell_start, cell_end, nl, ctl,
                                              gate);
}

void launch_step(const SimParams* dp, const WallOp* ops, WallGrid wg, const StateBuf& in_plain,
                 const StateBuf& in_sorted, const StateBuf& out, const OrderBuf& ob, int n_max,
                 NbrList nl, StepCtl* ctl, StepLink link, bool spin_free,
                 const ForceCapture* cap, double* eb, bool fast, cudaStream_t st) {
  const ForceCapture c = cap ? *cap : ForceCapture{};
  const int g = blocks(n_max);
#define BLAZE_STEP_ARGS dp, ops, wg, in_plain, in_sorted, out, ob, n_max, nl, ctl, link, c, eb
#define BLAZE_STEP(C, S, E) k_step<C, S, E, false><<<g, kThreads, 0, st>>>(BLAZE_STEP_ARGS)
#define BLAZE_STEP_FAST(C, S) k_step<C, S, false, true><<<g, kThreads, 0, st>>>(BLAZE_STEP_ARGS)
  if (fast && !eb) {
    if (cap) {
      if (spin_free) BLAZE_STEP_FAST(true, false);
      else BLAZE_STEP_FAST(true, true);
    } else {
      if (spin_free) BLAZE_STEP_FAST(false, false);
      else BLAZE_STEP_FAST(false, true);
    }
  } else if (eb) {
    if (cap) {
      if (spin_free) BLAZE_STEP(true, false, true);
      else BLAZE_STEP(true, true, true);
    } else {
      if (spin_free) BLAZE_STEP(false, false, true);
      else BLAZE_STEP(false, true, true);
    }
  } else if (cap) {
    if (spin_free) BLAZE_STEP(true, false, false);
    else BLAZE_STEP(true, true, false);
  } else {
    if (spin_free) BLAZE_STEP(false, false, false);
    else BLAZE_STEP(false, true, false);
  }
#undef BLAZE_STEP
#undef BLAZE_STEP_FAST
#undef BLAZE_STEP_ARGS
}

void launch_check_div(long long n, unsigned long long seed, unsigned long long* bad,
                      cudaStream_t st) {
  k_check_div<<<148 * 8, 256, 0, st>>>(n, seed, bad);
}

void launch_energy_reduce(const double* eb, int n_max, const StepCtl* ctl, double* part,
                          double* tally, cudaStream_t st) {
  const int nb = (n_max + kEnergyBlock - 1) / kEnergyBlock;
  k_energy_partial<<<nb, kEnergyBlock, 0, st>>>(eb, n_max, ctl, part);
  k_energy_final<<<1, kEnergyBlock, 0, st>>>(part, nb, tally);
}

void launch_move_dobj(SimParams* dp, int turn, float about_x, float about_y, float c, float s,
                      int translate, int n_dobj, cudaStream_t st) {
  if (n_dobj > 0) k_move_dobj<<<1, 32, 0, st>>>(dp, turn, about_x, about_y, c, s, translate);
}

void launch_rotate_wobj(WallOp* ops, int n_ops, uint32_t rot_mask, float about_x, float about_y,
                        float c, float s, cudaStream_t st) {
  if (n_ops > 0)
    k_rotate_wobj<<<(n_ops + 127) / 128, 128, 0, st>>>(ops, n_ops, rot_mask, about_x, about_y, c,
                                                        s);
}

void launch_pack_state(const SimParams* dp, const HostStage& hs, bool has_vel, bool has_avel,
                       const StateBuf& s, int* pid_dst, int* lift_dst, float4* ornt_dst,
                       bool has_ornt, int n, cudaStream_t st) {
  k_pack_state<<<blocks(n), kThreads, 0, st>>>(dp, hs, has_vel ? 1 : 0, has_avel ? 1 : 0, s,
                                               pid_dst, lift_dst, ornt_dst, has_ornt ? 1 : 0, n);
}

void launch_unpack_state(const SimParams* dp, const HostStage& hs, const StateBuf& s,
                         const int* pid_src, const float4* ornt_src, int n, cudaStream_t st) {
  k_unpack_state<<<blocks(n), kThreads, 0, st>>>(dp, hs, s, pid_src, ornt_src, n);
}

void launch_count_above(const float4* pos, const StepCtl* ctl, int n_max, float height,
                        unsigned int* out, cudaStream_t st) {
  k_count_above<<<blocks(n_max), kThreads, 0, st>>>(pos, ctl, n_max, height, out);
}

void launch_kill(const StateBuf& s, const OrderBuf& ob, int n_max, float kill_height,
                 int rotating, float3 max_size, StepCtl* ctl, cudaStream_t st) {
  k_kill<<<blocks(n_max), kThreads, 0, st>>>(s, ob, n_max, kill_height, rotating, max_size, ctl);
}

}  // namespace blaze
