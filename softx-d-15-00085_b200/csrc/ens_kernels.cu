// ens_kernels.cu -- kernels of the ensemble path (see ens_kernels.cuh).
//
//   k_ens_hash     system-prefixed cell key per particle
//   [radix sort, radix_sort.cu]
//   k_ens_reorder  gather state, pid and wall history into sorted order + cell table
//   k_ens_nlist    27-cell Verlet list inside the particle's own system, carrying
//                  the tangential history of every surviving contact by partner pid
//   k_ens_epoch    one thread: the new list becomes current
//   k_ens_step     pair law + walls + symplectic Euler, fused, gather only
//
// The contact model (per pair, with m* = ma mb / (ma + mb), R* = ra rb / (ra + rb),
// overlap d, unit normal n from b to a, v_n = (va - vb) . n):
//   linear        f_n = kn d - c_n v_n,  c_n = 2 beta sqrt(m* kn);  k_t = kt,
//                 c_t = 2 beta sqrt(m* kt)
//   Hertz-Mindlin S_n = 2 E* sqrt(R* d), f_n = 2/3 S_n d - c_n v_n,
//                 c_n = 2 sqrt(5/6) beta sqrt(S_n m*);  k_t = 8 G* sqrt(R* d),
//                 c_t = 2 sqrt(5/6) beta sqrt(k_t m*)
//   with beta = -ln e / sqrt(ln^2 e + pi^2); f_n is not clamped (the damping
//   may pull at the end of a contact, so the linear law rebounds with e).
//   Tangential: the history xi is turned into the tangent plane (length
//   kept), advanced by v_t dt, f_t = -k_t xi - c_t v_t, capped at
//   mu max(f_n, 0) (xi then set back to the spring length that gives the
//   capped force).  Rolling friction: a torque -mu_r max(f_n, 0) R* w_rel / |w_rel|.
//   Walls use the same law with R* = r, m* = m.
#include "ens_kernels.cuh"
#include "ens_device.cuh"
#include "dem_laws.cuh"

#include <algorithm>

namespace blaze {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------- hash
__global__ void __launch_bounds__(kThreads)
k_ens_hash(EnsGeom g, const float4* __restrict__ pos, const float4* __restrict__ vel, int n,
           uint32_t* __restrict__ keys, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t sys = __float_as_uint(vel[i].w) & kSysMask;
  const EnsSysDev& S = g.sys[sys];
  const int3 c = ens_cell(S, xyz(pos[i]));
  uint32_t st = 0, key;
  if (ens_in(S, c)) {
    key = ens_key(S, c);
  } else {
    key = g.ncell_tab;
    st = kStatusOutOfGrid;
  }
  keys[i] = key;
  ens_flag(ctl, st);
}

// ---------------------------------------------------------------- reorder
__global__ void __launch_bounds__(kThreads)
k_ens_reorder(StateBuf src, StateBuf dst, EnsBufs b, int n, const uint32_t* __restrict__ keys,
              const int32_t* __restrict__ perm, uint32_t* __restrict__ cstart,
              uint32_t* __restrict__ cend, uint32_t ncell_tab, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = ctl->epoch & 1;
  const int j = perm[i];
  const float4 x = src.pos[j];
  dst.pos[i] = x;
  const float4 v = src.vel[j];
  dst.vel[i] = v;
  float4 w = src.angv[j];
  if (x.w < 0.0f) {   // a polyhedron: angv.w is its id; its path restarts per id
    const int pq = __float_as_int(w.w);
    b.pat[pq] = i;
    b.ppath[pq] = 0.0f;
  } else {
    w.w = 0.0f;
  }
  dst.angv[i] = w;
  b.pid[e ^ 1][i] = b.pid[e][j];
  if ((__float_as_uint(v.w) >> kSysBits) != 0u) {
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      b.wh[e ^ 1][(size_t)q * b.stride + i] = b.wh[e][(size_t)q * b.stride + j];
  }
  const uint32_t k = keys[i];
  if (k < ncell_tab) {
    if (i == 0 || keys[i - 1] != k) cstart[k] = (uint32_t)i;
    if (i == n - 1 || keys[i + 1] != k) cend[k] = (uint32_t)i + 1u;
  }
}

// ------------------------------------------------------------------ nlist
// Pairs with |xi - xj|^2 < (ri + rj + skin)^2 from the 27 surrounding cells
// of the particle's own system (z, y, x order; j ascending inside a cell).
// The history of a slot of the old list moves to the new slot of the same
// partner (matched by pid).
__global__ void __launch_bounds__(kThreads)
k_ens_nlist(EnsGeom g, EnsBufs b, const float4* __restrict__ pos, const float4* __restrict__ vel,
            int n, const int32_t* __restrict__ perm, const uint32_t* __restrict__ cstart,
            const uint32_t* __restrict__ cend, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = ctl->epoch & 1;
  const EnsList Lo = b.L[e], Ln = b.L[e ^ 1];
  const int* pid_old = b.pid[e];
  const int* pid_new = b.pid[e ^ 1];
  const size_t stride = (size_t)b.stride;
  const float4 pa4 = pos[i];
  if (pa4.w < 0.0f) {   // a polyhedron: its neighbours are listed by k_mix_plist
    Ln.cnt[i] = 0;
    Ln.mask[i] = 0;
    return;
  }
  const float3 pa = xyz(pa4);
  const float ra = pa4.w;
  const uint32_t sys = __float_as_uint(vel[i].w) & kSysMask;
  const EnsSysDev& S = g.sys[sys];
  const int3 c = ens_cell(S, pa);
  const int io = perm[i];
  const uint32_t cnt_o = Lo.cnt[io];
  const uint32_t mask_o = Lo.mask[io];
  uint32_t cnt = 0, mask = 0, st = 0;
  if (ens_in(S, c)) {
    const int x0 = c.x > 0 ? c.x - 1 : 0, x1 = c.x < S.nc.x - 1 ? c.x + 1 : c.x;
    const int y0 = c.y > 0 ? c.y - 1 : 0, y1 = c.y < S.nc.y - 1 ? c.y + 1 : c.y;
    const int z0 = c.z > 0 ? c.z - 1 : 0, z1 = c.z < S.nc.z - 1 ? c.z + 1 : c.z;
    for (int z = z0; z <= z1; ++z)
      for (int y = y0; y <= y1; ++y) {
        const uint32_t row = S.cell_off + (uint32_t)(S.nc.x * (y + S.nc.y * z));
        for (int x = x0; x <= x1; ++x) {
          const uint32_t h = row + (uint32_t)x;
          const uint32_t s = __ldg(cstart + h);
          if (s == 0xffffffffu) continue;
          const uint32_t eo = __ldg(cend + h);
          for (uint32_t j = s; j < eo; ++j) {
            if ((int)j == i) continue;
            const float4 pb = __ldg(pos + j);
            const float3 rel = pa - xyz(pb);
            const float lim = (ra + fabsf(pb.w)) + g.skin;   // a polyhedron: its bounding radius
            if (!(dot3(rel, rel) < lim * lim)) continue;
            if (cnt < (uint32_t)b.cap) {
              Ln.idx[cnt * stride + i] = j;
              uint8_t from = 0xffu;
              uint32_t mo = mask_o;
              if (mo) {
                const int pj = pid_new[j];
                while (mo) {
                  const int ko = __ffs(mo) - 1;
                  mo &= mo - 1u;
                  if ((uint32_t)ko >= cnt_o) break;
                  const size_t so = (size_t)ko * stride + io;
                  if (pid_old[Lo.idx[so]] == pj) {
                    const size_t sn = (size_t)cnt * stride + i;
                    Ln.hx[sn] = Lo.hx[so];
                    Ln.hy[sn] = Lo.hy[so];
                    Ln.hz[sn] = Lo.hz[so];
                    mask |= 1u << cnt;
                    from = (uint8_t)ko;
                    break;
                  }
                }
              }
              if (Ln.src) Ln.src[cnt * stride + i] = from;
            } else {
              st |= kStatusListOverflow;
            }
            ++cnt;
          }
        }
      }
  } else {
    st |= kStatusOutOfGrid;
  }
  Ln.cnt[i] = cnt < (uint32_t)b.cap ? cnt : (uint32_t)b.cap;
  Ln.mask[i] = mask;
  ens_flag(ctl, st);
}

__global__ void k_ens_epoch(StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  ctl->epoch += 1;
}

// ------------------------------------------------------------------- step
// candidate slots tested per batch of independent loads in the contact pass
constexpr uint32_t kEnsMaskBatch = 4;
// A neighbour's state: through the read-only cache (kNc) when the state
// cannot change during the kernel, else a plain load (the persistent kernel
// reads, after a grid barrier, what other blocks wrote in the same launch).
template <bool kNc>
__device__ __forceinline__ float4 ld_state(const float4* p) {
  if constexpr (kNc) return __ldg(p);
  else return *p;
}

// ----------------------------------------------------- reference law (3)
// The reference's sphere step, per particle, with the parameters its
// parser derives for a particle object formed here from the particle's own
// radius and the system's constants:
//   mass     m = (4/3 pi density) r^3 in double, rounded once
//            (KSimulationData.cpp:1096); 1/I = 1 / (0.4 r r m) in float
//            (main.cpp:622-626)
//   pairs    Kn = kn, Cn = (ref_a sqrt(Kn m*)) / ref_b in double with
//            m* = 1 / (1/ma + 1/mb) (KSimulationData.cpp:955-1016), kinetic
//            friction mu
//   planes   Kn = kn, Cn the same with m* = m (KSimulationData.cpp:1019-1047),
//            static friction mu_wall
// The contact test and penetration (|d| - (ra + rb), plus 1e-5), the laws
// (Collision_Response.cuh:374-494 and 4-109) and the integration
// (Integrate_Euler_NonSymmetry, Integration.cuh:6-184, rolling resistance
// mu_roll) are the sphere path's own functions; a plane is tested as the
// reference tests a face (Collision_Detection_Spheres.cuh:6-100) against
// its point d n.  The law keeps no history.
__device__ __forceinline__ float ref_mass(const EnsSysDev& S, float r) {
  const double r3 = ((double)r * (double)r) * (double)r;
  return (float)(S.ref_m * r3);
}

__device__ __forceinline__ float ref_damping(const EnsSysDev& S, double m) {
  return S.ref_b > 0.0 ? (float)((S.ref_a * sqrt((double)S.kn * m)) / S.ref_b) : 0.0f;
}

template <bool kCapture, bool kNc>
__device__ __forceinline__ float ens_particle_step_ref(const EnsGeom& g, const EnsBufs& b,
                                                       const StateBuf& in, const StateBuf& out,
                                                       int i, const EnsList& L,
                                                       const EnsCapture& cap, uint32_t& st) {
  const size_t stride = (size_t)b.stride;
  const float dt = g.dt;
  const float4 pa4 = in.pos[i], va4 = in.vel[i], wa4 = in.angv[i];
  const float3 pa = xyz(pa4), va = xyz(va4), wa = xyz(wa4);
  const float ra = pa4.w;
  const uint32_t sys = __float_as_uint(va4.w) & kSysMask;
  const EnsSysDev& S = g.sys[sys];
  const float ma = ref_mass(S, ra);
  SimParams P;   // the two fields the reference's laws read
  P.dt = dt;
  P.rotation = 1;

  // particle-particle (Kernel_ParticleInteraction_Spheres_NonSymmetry)
  float3 f = S.gravity * ma;
  float3 tl = f3(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = L.cnt[i];
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = L.idx[(size_t)k * stride + i];
    const float4 pb4 = ld_state<kNc>(in.pos + j);
    const float3 rel = pa - xyz(pb4);
    const float rb = pb4.w;
    if (!touches(rel, ra + rb)) continue;
    const float dist = len3(rel);
    const float dis = fabsf(dist - (ra + rb)) + 0.000010f;
    const float3 nrm = div3_rn(rel, dist);
    const float4 vb4 = ld_state<kNc>(in.vel + j), wb4 = ld_state<kNc>(in.angv + j);
    const float mb = ref_mass(S, rb);
    PP_Parms pp;
    pp.Kn = S.kn;
    pp.Cn = ref_damping(S, 1.0 / ((1.0 / (double)ma) + (1.0 / (double)mb)));
    pp.Fric_static = S.mu;
    pp.Fric_kinetic = S.mu;
    const Forces F = law_pp<true>(P, va - xyz(vb4), nrm, dis, (-1.0f * nrm) * ra, nrm * rb, wa,
                                  xyz(wb4), pp, va, xyz(vb4), ma, mb);
    f = f + F.trans;
    tl = tl + F.torque;
  }

  // plane walls (WorldObject_InteractionParticle, face and plane contacts)
  float3 fw = f3(0.0f, 0.0f, 0.0f), tw = f3(0.0f, 0.0f, 0.0f);
  TypeParams T;
  T.mass = ma;
  T.s_kn = S.kn;
  T.s_cn = ref_damping(S, (double)ma);
  T.s_mus = S.mu_w;
  for (int w = S.wall0; w < S.wall0 + S.nwall; ++w) {
    const EnsWallDev& W = g.walls[w];
    const float3 n = W.a;
    const float3 c = n * W.r;
    const float3 pt = pa - ra * n;
    float dis = dot3(n, pt - c);
    if (!(dis < 0.000000f && dis > -ra)) continue;
    dis = fabsf(dis);
    const Forces F = law_static_surface(P, va, n, dis, pt - pa, wa, T);
    fw = fw + F.trans;
    tw = tw + F.torque;
  }

  // Integrate_Euler_NonSymmetry (Integration.cuh:6-184), spheres
  float3 acc = fw + f;
  acc = acc * (1.0f / ma);
  const float3 v = va + acc * dt;
  const float3 p = pa + v * dt;
  const float3 tq = tl + tw;
  float3 w = wa;
  if (dot3(tq, tq) > 0.0f) {
    const float iinv = 1.0f / (((0.4f * ra) * ra) * ma);
    const float3 aa = iinv * tq;
    w = w + aa * dt;
    w = w - w * S.mu_r;
  }
  const float path = wa4.w + len3(v) * dt;
  out.pos[i] = make_float4(p.x, p.y, p.z, ra);
  out.vel[i] = make_float4(v.x, v.y, v.z, __uint_as_float(sys));
  out.angv[i] = make_float4(w.x, w.y, w.z, path);
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) st |= kStatusNonFinite;
  if (kCapture) {
    const float3 fc = (f - S.gravity * ma) + fw;
    cap.f[i] = make_float4(fc.x, fc.y, fc.z, 0.0f);
    cap.t[i] = make_float4(tq.x, tq.y, tq.z, 0.0f);
  }
  return path;
}


// The step of particle i: its contacts in list order (tangential histories
// updated in place, the particle's own slots only), its walls, symplectic
// Euler from `in` into `out`.  Raises status bits in st; returns the path
// the particle has moved since the last re-sort.  kRecord: also writes what
// the step reads into the tape view (histories to hrec when it is not null).
// kMix: the system holds polyhedra (linear law): a polyhedron's own entry is
// skipped (k_mix_poly_step steps it); a polyhedron neighbour's contact force
// and torque are the ones k_mix_poly_step left for this sphere (MixView),
// added in slot order.
template <int kLaw, bool kCapture, bool kRecord, bool kCurved, bool kNc = true, bool kRot = false,
          bool kMix = false>
__device__ __forceinline__ float ens_particle_step(const EnsGeom& g, const EnsBufs& b,
                                                   const StateBuf& in, const StateBuf& out,
                                                   int i, int e, const EnsList& L, TapeView tv,
                                                   float* hrec, const EnsCapture& cap,
                                                   uint32_t& st) {
  if constexpr (kLaw == kLawReference) {
    return ens_particle_step_ref<kCapture, kNc>(g, b, in, out, i, L, cap, st);
  } else {
  const size_t stride = (size_t)b.stride;
  const float dt = g.dt;
  const float4 pa4 = in.pos[i], va4 = in.vel[i], wa4 = in.angv[i];
  if constexpr (kMix) {
    if (pa4.w < 0.0f) return 0.0f;
  }
  const float3 pa = xyz(pa4), va = xyz(va4), wa = xyz(wa4);
  const float ra = pa4.w;
  const uint32_t bits = __float_as_uint(va4.w);
  const uint32_t sys = bits & kSysMask;
  const uint32_t wmask_o = bits >> kSysBits;
  const EnsSysDev& S = g.sys[sys];
  const float ma = sphere_mass(S, ra);

  // particle-particle contacts, in list order
  float3 f = f3(0.0f, 0.0f, 0.0f), t = f3(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = L.cnt[i];
  const uint32_t mask_o = L.mask[i];
  if constexpr (kRecord) {
    tv.pos[i] = pa4;
    tv.vel[i] = va4;
    tv.angv[i] = wa4;
    tv.mask[i] = mask_o;
  }
  uint32_t mask = 0;
  // contacts first, candidates in batches (all index loads of a batch, then
  // all position gathers, then the tests); then the law over the contacts
  // alone, in list order
  uint32_t cmask = 0;
  for (uint32_t k0 = 0; k0 < cnt; k0 += kEnsMaskBatch) {
    uint32_t jj[kEnsMaskBatch];
#pragma unroll
    for (uint32_t u = 0; u < kEnsMaskBatch; ++u)
      jj[u] = k0 + u < cnt ? __ldg(L.idx + (size_t)(k0 + u) * stride + i) : 0u;
    float4 pb[kEnsMaskBatch];
#pragma unroll
    for (uint32_t u = 0; u < kEnsMaskBatch; ++u)
      pb[u] = k0 + u < cnt ? ld_state<kNc>(in.pos + jj[u]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (uint32_t u = 0; u < kEnsMaskBatch; ++u) {
      const float3 rel = pa - xyz(pb[u]);
      const float sr = ra + (kMix ? fabsf(pb[u].w) : pb[u].w);
      const float d2 = dot3(rel, rel);
      if (k0 + u < cnt && d2 < sr * sr && sqrtf(d2) > 0.0f) cmask |= 1u << (k0 + u);
    }
  }
  // the contacts in slot order.  On a turning drum the next contact's slot
  // and gathers are issued before this contact's law (measured: mill mesh
  // -6 %, mixed charge -2 % a step); the static silo and the plane-walled
  // boxes ran faster without (+4 % and +1 % with it: more registers)
  constexpr bool kPipe = kRot;
  uint32_t kn = 0u, jn = 0u;
  float4 pn4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), vn4 = pn4, wn4 = pn4;
  bool more = cmask != 0u;
  if (kPipe && more) {
    kn = (uint32_t)(__ffs(cmask) - 1);
    cmask &= cmask - 1u;
    jn = L.idx[(size_t)kn * stride + i];
    pn4 = ld_state<kNc>(in.pos + jn);
    vn4 = ld_state<kNc>(in.vel + jn);
    wn4 = ld_state<kNc>(in.angv + jn);
  }
  while (more) {
    uint32_t k, j;
    float4 pb4, vb4, wb4;
    if constexpr (kPipe) {
      k = kn;
      j = jn;
      pb4 = pn4;
      vb4 = vn4;
      wb4 = wn4;
      more = cmask != 0u;
      if (more) {
        kn = (uint32_t)(__ffs(cmask) - 1);
        cmask &= cmask - 1u;
        jn = L.idx[(size_t)kn * stride + i];
        pn4 = ld_state<kNc>(in.pos + jn);
        vn4 = ld_state<kNc>(in.vel + jn);
        wn4 = ld_state<kNc>(in.angv + jn);
      }
    } else {
      k = (uint32_t)(__ffs(cmask) - 1);
      cmask &= cmask - 1u;
      more = cmask != 0u;
      j = L.idx[(size_t)k * stride + i];
      pb4 = ld_state<kNc>(in.pos + j);
    }
    const size_t sk = (size_t)k * stride + i;
    if constexpr (kMix) {
      if (pb4.w < 0.0f) {
        const uint32_t tw = g.mix.twin[sk];
        if (tw == 0xffu) continue;
        const int q = __float_as_int(kPipe ? wb4.w : ld_state<kNc>(in.angv + j).w);
        const size_t sq = (size_t)tw * (size_t)g.mix.npoly + (size_t)q;
        const float4 F4 = g.mix.sf[sq];
        if (F4.w == 0.0f) continue;
        const float4 T4 = g.mix.st[sq];
        f = f + xyz(F4);
        t = t + xyz(T4);
        continue;
      }
    }
    const float3 rel = pa - xyz(pb4);
    const float rb = pb4.w;
    const float sr = ra + rb;
    const float d2 = dot3(rel, rel);
    if (!(d2 < sr * sr)) continue;
    const float dist = sqrtf(d2);
    if (!(dist > 0.0f)) continue;
    const float3 nrm = rel * (1.0f / dist);
    // the contact is decided by the overlap itself: the FP32 test above can
    // pass a pair whose FP64-formed overlap is not positive
    const float delta = overlap_pair(ra, rb, pa, xyz(pb4));
    if (!(delta > 0.0f)) continue;
    if constexpr (!kPipe) {
      vb4 = ld_state<kNc>(in.vel + j);
      wb4 = ld_state<kNc>(in.angv + j);
    }
    const float3 vb = xyz(vb4), wb = xyz(wb4);
    const float mb = sphere_mass(S, rb);
    float3 xi = f3(0.0f, 0.0f, 0.0f);
    if ((mask_o >> k) & 1u) {
      xi = f3(L.hx[sk], L.hy[sk], L.hz[sk]);
      if constexpr (kRecord) {
        if (hrec) {
          float* h = hrec + 3 * __popc(mask_o & ((1u << k) - 1u));
          h[0] = xi.x;
          h[1] = xi.y;
          h[2] = xi.z;
        }
      }
    }
    const float rs = (ra * rb) / (ra + rb);
    const float ms = (ma * mb) / (ma + mb);
    const float3 vcpa = va + cross3(wa, nrm * (-ra));
    const float3 vcpb = vb + cross3(wb, nrm * rb);
    float3 F, T;
    contact_law<kLaw>(S, S.mu, nrm, delta, rs, ms, va - vb, vcpa - vcpb, wa - wb, ra, dt, xi,
                      F, T);
    L.hx[sk] = xi.x;
    L.hy[sk] = xi.y;
    L.hz[sk] = xi.z;
    mask |= 1u << k;
    f = f + F;
    t = t + T;
  }
  if (mask != mask_o) L.mask[i] = mask;
  if constexpr (kRecord) tv.cmask[i] = mask;

  // walls: old history slots (by wall id) held in registers; new slots are
  // written in processing order straight over the old ones
  float4 oh[kWallSlots];
#pragma unroll
  for (int q = 0; q < kWallSlots; ++q) oh[q] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
  if (wmask_o) {
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      if ((wmask_o >> q) & 1u) oh[q] = b.wh[e][(size_t)q * stride + i];
    if constexpr (kRecord) {
      if (hrec) {
        float* h = hrec + 3 * __popc(mask_o);
#pragma unroll
        for (int q = 0; q < kWallSlots; ++q)
          if ((wmask_o >> q) & 1u) {
            float* hq = h + 4 * __popc(wmask_o & ((1u << q) - 1u));
            hq[0] = oh[q].x;
            hq[1] = oh[q].y;
            hq[2] = oh[q].z;
            hq[3] = oh[q].w;
          }
      }
    }
  }
  int nw = 0;
  // a turning drum (kCurved only): its triangles are tested in the drum's
  // frame, where they stand still, and the normals turned back; triangles
  // and cylinders move with the turn
  bool rot = false;
  float rc = 1.0f, rsn = 0.0f;
  if constexpr (kCurved && kRot) {
    if (S.rot) {
      rot = true;
      const float2 cs = g.rot[sys];
      rc = cs.x;
      rsn = cs.y;
    }
  }
  auto wall_contact = [&](int id, float3 nrm, float delta, bool moving) {
    float3 xi = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      if (__float_as_int(oh[q].w) == id) xi = f3(oh[q].x, oh[q].y, oh[q].z);
    const float3 vcpa = va + cross3(wa, nrm * (-ra));
    float3 vr = va, vc = vcpa, wr = wa;
    if (moving) {
      // the wall's velocity at the contact point, and its spin
      const float3 vw = cross3(S.rot_a, (pa - nrm * ra) - S.rot_o) * S.rot_w;
      vr = va - vw;
      vc = vcpa - vw;
      wr = wa - S.rot_a * S.rot_w;
    }
    float3 F, T;
    contact_law<kLaw>(S, S.mu_w, nrm, delta, ra, ma, vr, vc, wr, ra, dt, xi, F, T);
    f = f + F;
    t = t + T;
    if (nw < kWallSlots) {
      b.wh[e][(size_t)nw * stride + i] = make_float4(xi.x, xi.y, xi.z, __int_as_float(id));
      ++nw;
    } else {
      st |= kStatusListOverflow;
    }
  };
  for (int w = S.wall0; w < S.wall0 + S.nwall; ++w) {
    const EnsWallDev& W = g.walls[w];
    float3 nrm;
    float delta;
    int region;
    if (wall_touch<kCurved>(W, pa, ra, nrm, delta, region))
      wall_contact(w, nrm, delta, rot && W.turning);
  }
  if (kCurved && g.tri_off) {
    const float3 pd = rot ? S.rot_o + rot_about(S.rot_a, rc, -rsn, pa - S.rot_o) : pa;
    const int3 c = ens_scell(S, pd);
    if (ens_sin(S, c)) {
      const uint32_t h = ens_skey(S, c);
      const uint32_t o0 = __ldg(g.stri_off + h), o1 = __ldg(g.stri_off + h + 1);
      // face contacts all count; without one, only the deepest edge/vertex
      // contact does (a sphere over a shared edge or vertex touches it once)
      int nface = 0, best = -1;
      float best_d = 0.0f;
      for (uint32_t q = o0; q < o1; ++q) {
        const int id = (int)__ldg(g.stri_ids + q);
        float3 nrm;
        float delta;
        int region;
        if (!wall_touch<kCurved>(g.walls[id], pd, ra, nrm, delta, region)) continue;
        if (region == 0) ++nface;
        else if (best < 0 || delta > best_d) { best = id; best_d = delta; }
      }
      for (uint32_t q = o0; q < o1; ++q) {
        const int id = (int)__ldg(g.stri_ids + q);
        float3 nrm;
        float delta;
        int region;
        if (!wall_touch<kCurved>(g.walls[id], pd, ra, nrm, delta, region)) continue;
        if ((nface > 0 && region == 0) || (nface == 0 && id == best))
          wall_contact(id, rot ? rot_about(S.rot_a, rc, rsn, nrm) : nrm, delta, rot);
      }
    }
  }
  const uint32_t wmask = nw >= kWallSlots ? (1u << kWallSlots) - 1u : (1u << nw) - 1u;

  // symplectic Euler
  const float inv_m = 1.0f / ma;
  const float3 acc = f * inv_m + S.gravity;
  const float3 v = va + acc * dt;
  const float3 p = pa + v * dt;
  const float inertia = (0.4f * ma) * (ra * ra);
  const float3 w = wa + (t * (1.0f / inertia)) * dt;
  const float path = wa4.w + len3(v) * dt;
  out.pos[i] = make_float4(p.x, p.y, p.z, ra);
  out.vel[i] = make_float4(v.x, v.y, v.z, __uint_as_float(sys | (wmask << kSysBits)));
  out.angv[i] = make_float4(w.x, w.y, w.z, path);
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) st |= kStatusNonFinite;
  if (kCapture) {
    cap.f[i] = make_float4(f.x, f.y, f.z, 0.0f);
    cap.t[i] = make_float4(t.x, t.y, t.z, 0.0f);
  }
  return path;
  }
}

// kRecord: also write what the step reads into tape slot tp.ctl->slot (the
// history words are reserved first, by every thread of the block).
template <int kLaw, bool kCapture, bool kRecord, bool kCurved, bool kRot, bool kMix>
__device__ __forceinline__ void ens_step_body(const EnsGeom& g, const EnsBufs& b,
                                              const StateBuf& in_plain, const StateBuf& in_sorted,
                                              const StateBuf& out, int n, StepCtl* ctl,
                                              const StepLink& link, const EnsCapture& cap,
                                              const EnsTape& tp) {
  const bool rebuilt = *link.rebuilt != 0;
  const StateBuf in = rebuilt ? in_sorted : in_plain;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = ctl->epoch & 1;
  const EnsList L = b.L[e];
  TapeView tv{};
  float* hrec = nullptr;
  if constexpr (kRecord) {
    const TapeStep ts = tp.steps[tp.ctl->slot];
    tv = tape_view(tp, ts.block, n);
    uint32_t words = 0;
    if (i < n)
      words = 3u * (uint32_t)__popc(L.mask[i]) +
              4u * (uint32_t)__popc(__float_as_uint(in.vel[i].w) >> kSysBits);
    bool ok;
    const uint32_t off =
        tape_reserve(words, &tp.ctl->cur, tp.ctl->lim, ts.hbase, &tp.ctl->overflow, ok);
    if (i < n) {
      tv.hoff[i] = off;
      if (ok) hrec = reinterpret_cast<float*>(tp.arena + ts.hbase + off);
    }
  }
  if (i >= n) return;
  uint32_t st = 0;
  const float path =
      ens_particle_step<kLaw, kCapture, kRecord, kCurved, true, kRot, kMix>(g, b, in, out, i, e, L,
                                                                             tv, hrec, cap, st);
  {
    const unsigned m = __activemask();
    const unsigned req = __ballot_sync(m, path > 0.5f * g.skin);
    if (req && (threadIdx.x & 31) == (__ffs(m) - 1)) {
      if (link.has_next_h) cudaGraphSetConditional(link.next_h, 1u);
      else atomicExch(&ctl->rebuild_req, 1);
    }
  }
  ens_flag(ctl, st);
}

template <int kLaw, bool kCapture, bool kRecord, bool kCurved, bool kRot = false,
          bool kMix = false>
__global__ void __launch_bounds__(kMaxStepBlock)
k_ens_step(EnsGeom g, EnsBufs b, StateBuf in_plain, StateBuf in_sorted, StateBuf out, int n,
           StepCtl* ctl, StepLink link, EnsCapture cap, EnsTape tp) {
  ens_step_body<kLaw, kCapture, kRecord, kCurved, kRot, kMix>(g, b, in_plain, in_sorted, out, n,
                                                             ctl, link, cap, tp);
}

// The recording step (reverse mode, linear law, plane walls) held to the
// plain step's 80 registers: at the 88 it takes by itself a block of 256
// fits twice per SM instead of three times.
constexpr int kRecordRegs = 80;
__global__ void __maxnreg__(kRecordRegs)
k_ens_step_rec(EnsGeom g, EnsBufs b, StateBuf in_plain, StateBuf in_sorted, StateBuf out, int n,
               StepCtl* ctl, StepLink link, EnsTape tp) {
  ens_step_body<kLawLinear, false, true, false, false, false>(
      g, b, in_plain, in_sorted, out, n, ctl, link, EnsCapture{nullptr, nullptr}, tp);
}

// ------------------------------------------------------------ drum turn
__global__ void k_ens_rot_tick(const EnsSysDev* __restrict__ sys, float2* rot, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || !sys[s].rot) return;
  const float2 r = rot[s];
  const float c1 = r.x * sys[s].rot_cd - r.y * sys[s].rot_sd;
  const float s1 = r.y * sys[s].rot_cd + r.x * sys[s].rot_sd;
  const float m = sqrtf(c1 * c1 + s1 * s1);
  rot[s] = make_float2(c1 / m, s1 / m);
}

// ------------------------------------------------------- persistent steps
// One launch runs up to *left steps with a grid barrier between them, so a
// stretch of steps without a re-sort costs one launch instead of one launch
// and one conditional node per step.  Every block is resident (cooperative
// launch, grid from the occupancy), the particles are strided over the grid.
// Buffers: step 0 reads the sorted copy after a re-sort, else `home`; steps
// then alternate home -> other -> home, and an odd count ends with a copy
// back, so each launch leaves the state in `home`.  A step whose particles
// ask for a re-sort is the launch's last: requests record the step index
// (atomicMin), and after barrier k every block reads the same answer to
// "was one made at step <= k" (a block already in step k + 1 can only write
// k + 1).  Barrier waits are bounded by the global timer; a block that gives
// up raises kStatusTimeout and the abort word, and every block returns.
constexpr unsigned long long kBarrierLimitNs = 2000000000ull;   // 2 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Arrival counter bar[0], generation bar[1], abort word bar[2].  Returns
// false when the barrier was aborted (by this block or another).
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks,
                                             StepCtl* ctl) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vb = bar;
    int ok = vb[2] == 0u;
    if (ok) {
      const unsigned int gen = vb[1];
      __threadfence();
      if (atomicAdd(bar, 1u) == nblocks - 1u) {
        atomicExch(bar, 0u);
        __threadfence();
        atomicAdd(bar + 1, 1u);
      } else {
        const unsigned long long t0 = global_ns();
        while (vb[1] == gen) {
          if (vb[2] != 0u) { ok = 0; break; }
          if (global_ns() - t0 > kBarrierLimitNs) {
            atomicExch(bar + 2, 1u);
            atomicOr(&ctl->status, kStatusTimeout);
            ok = 0;
            break;
          }
          __nanosleep(100);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Registers capped at the step kernel's count, so as many blocks stay
// resident as the per-step launches have.
constexpr int kPersistRegs = 80;

// Self-check of the barrier's bounded wait: the barrier is told of one
// block more than the launch has, so nothing completes it; every block must
// give up after the limit, raise kStatusTimeout and return.
__global__ void k_barrier_check(unsigned int* bar, StepCtl* ctl) {
  grid_barrier(bar, gridDim.x + 1u, ctl);
}

template <int kLaw, bool kCurved>
__global__ void __maxnreg__(kPersistRegs)
k_ens_persist(EnsGeom g, EnsBufs b, StateBuf home, StateBuf other, StateBuf sorted, int n,
              StepCtl* ctl, const int* rebuilt, EnsPersist p) {
  const int e = ctl->epoch & 1;
  const EnsList L = b.L[e];
  const int budget = *p.left;
  const bool rb = *rebuilt != 0;
  const int gstride = gridDim.x * blockDim.x;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  int done = 0;
  bool stop = false, aborted = false;
  for (int k = 0; k < budget && !stop; ++k) {
    const StateBuf in = k == 0 ? (rb ? sorted : home) : ((k & 1) ? other : home);
    const StateBuf out = (k & 1) ? home : other;
    uint32_t st = 0;
    bool req = false;
    for (int i = i0; i < n; i += gstride) {
      const float path = ens_particle_step<kLaw, false, false, kCurved, false>(
          g, b, in, out, i, e, L, TapeView{}, nullptr, EnsCapture{nullptr, nullptr}, st);
      req |= path > 0.5f * g.skin;
    }
    if (__syncthreads_or(req ? 1 : 0) && threadIdx.x == 0) atomicMin(p.req_step, k);
    if (st) atomicOr(&ctl->status, st);
    if (!grid_barrier(p.bar, gridDim.x, ctl)) { aborted = true; break; }
    done = k + 1;
    stop = *(volatile int*)p.req_step <= k;
  }
  if (!aborted && (done & 1)) {
    for (int i = i0; i < n; i += gstride) {
      home.pos[i] = other.pos[i];
      home.vel[i] = other.vel[i];
      home.angv[i] = other.angv[i];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int left = aborted ? 0 : budget - done;
    if (stop) ctl->rebuild_req = 1;
    if (aborted) left = 0;
    *p.left = left;
    *p.done += done;
    cudaGraphSetConditional(p.loop_h, left > 0 ? 1u : 0u);
  }
}

// Start of a round of the WHILE loop: take the pending re-sort request into
// the IF node, clear the round's words.
__global__ void k_ens_persist_gate(StepCtl* ctl, EnsPersist p, int* rb,
                                   cudaGraphConditionalHandle if_h) {
  const int r = ctl->rebuild_req;
  ctl->rebuild_req = 0;
  *rb = 0;
  *p.req_step = 0x7fffffff;
  p.bar[0] = 0u;
  p.bar[1] = 0u;
  p.bar[2] = 0u;
  cudaGraphSetConditional(if_h, r ? 1u : 0u);
}

__global__ void k_ens_persist_init(EnsPersist p, int steps) {
  *p.left = steps;
}

// ---------------------------------------------------------------- staging
__global__ void __launch_bounds__(kThreads)
k_ens_pack(const float* __restrict__ pos3, const float* __restrict__ rad,
           const float* __restrict__ vel3, const float* __restrict__ avel3,
           const int* __restrict__ sys_of, StateBuf s, int* __restrict__ pid, EnsList L0,
           EnsList L1, int n, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float r = rad[i];
  s.pos[i] = make_float4(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2], r);
  const float sb = __uint_as_float((uint32_t)sys_of[i] & kSysMask);
  s.vel[i] = vel3 ? make_float4(vel3[3 * i], vel3[3 * i + 1], vel3[3 * i + 2], sb)
                  : make_float4(0.0f, 0.0f, 0.0f, sb);
  s.angv[i] = avel3 ? make_float4(avel3[3 * i], avel3[3 * i + 1], avel3[3 * i + 2], 0.0f)
                    : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  pid[i] = i;
  L0.cnt[i] = 0; L0.mask[i] = 0;
  L1.cnt[i] = 0; L1.mask[i] = 0;
  if (!(r > 0.0f) || !isfinite(r)) atomicOr(flags, 1);
}

__global__ void __launch_bounds__(kThreads)
k_ens_unpack(StateBuf s, const int* __restrict__ pid_src, int n, float* pos3, float* rad,
             float* vel3, float* avel3, int* sys, int* pid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = s.pos[i], v = s.vel[i], w = s.angv[i];
  pos3[3 * i] = p.x; pos3[3 * i + 1] = p.y; pos3[3 * i + 2] = p.z;
  rad[i] = fabsf(p.w);   // a polyhedron: its bounding radius
  vel3[3 * i] = v.x; vel3[3 * i + 1] = v.y; vel3[3 * i + 2] = v.z;
  avel3[3 * i] = w.x; avel3[3 * i + 1] = w.y; avel3[3 * i + 2] = w.z;
  sys[i] = (int)(__float_as_uint(v.w) & kSysMask);
  pid[i] = pid_src[i];
}

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

void ens_launch_hash(const EnsGeom& g, const EnsBufs& b, int cur, int n, uint32_t* keys,
                     StepCtl* ctl, const int* gate, cudaStream_t st) {
  k_ens_hash<<<nblk(n), kThreads, 0, st>>>(g, b.S[cur].pos, b.S[cur].vel, n, keys, ctl, gate);
}

void ens_launch_reorder(const EnsBufs& b, int cur, int n, const uint32_t* keys,
                        const int32_t* perm, uint32_t* cstart, uint32_t* cend, uint32_t ncell_tab,
                        StepCtl* ctl, const int* gate, cudaStream_t st) {
  k_ens_reorder<<<nblk(n), kThreads, 0, st>>>(b.S[cur], b.S[2], b, n, keys, perm, cstart, cend,
                                              ncell_tab, ctl, gate);
}

void ens_launch_nlist(const EnsGeom& g, const EnsBufs& b, int n, const int32_t* perm,
                      const uint32_t* cstart, const uint32_t* cend, StepCtl* ctl,
                      const int* gate, cudaStream_t st) {
  k_ens_nlist<<<nblk(n), kThreads, 0, st>>>(g, b, b.S[2].pos, b.S[2].vel, n, perm, cstart, cend,
                                            ctl, gate);
}

void ens_launch_epoch(StepCtl* ctl, const int* gate, cudaStream_t st) {
  k_ens_epoch<<<1, 1, 0, st>>>(ctl, gate);
}

void ens_launch_step(const EnsGeom& g, const EnsBufs& b, int cur, int n, StepCtl* ctl,
                     StepLink link, const EnsCapture* cap, int block, cudaStream_t st) {
  const EnsCapture c = cap ? *cap : EnsCapture{nullptr, nullptr};
  const int bs = block >= 64 && block <= kMaxStepBlock && block % 32 == 0 ? block : kThreads;
  const int gs = (n + bs - 1) / bs;
#define ENS_ARGS g, b, b.S[cur], b.S[2], b.S[cur ^ 1], n, ctl, link, c, EnsTape{}
#define ENS_STEP(L, C, K) k_ens_step<L, C, false, K><<<gs, bs, 0, st>>>(ENS_ARGS)
#define ENS_STEP_ROT(L, C) k_ens_step<L, C, false, true, true><<<gs, bs, 0, st>>>(ENS_ARGS)
#define ENS_STEP_MIX(C, K, R) k_ens_step<kLawLinear, C, false, K, R, true><<<gs, bs, 0, st>>>(ENS_ARGS)
  if (g.mix.npoly > 0) {   // polyhedra among the spheres (linear law)
    if (g.curved && g.any_rot) {
      if (cap) ENS_STEP_MIX(true, true, true);
      else ENS_STEP_MIX(false, true, true);
    } else if (g.curved) {
      if (cap) ENS_STEP_MIX(true, true, false);
      else ENS_STEP_MIX(false, true, false);
    } else {
      if (cap) ENS_STEP_MIX(true, false, false);
      else ENS_STEP_MIX(false, false, false);
    }
  } else if (g.curved && g.any_rot) {   // a turning drum
    if (g.law == kLawHertz) {
      if (cap) ENS_STEP_ROT(kLawHertz, true);
      else ENS_STEP_ROT(kLawHertz, false);
    } else {
      if (cap) ENS_STEP_ROT(kLawLinear, true);
      else ENS_STEP_ROT(kLawLinear, false);
    }
  } else if (g.curved) {
    if (g.law == kLawHertz) {
      if (cap) ENS_STEP(kLawHertz, true, true);
      else ENS_STEP(kLawHertz, false, true);
    } else {
      if (cap) ENS_STEP(kLawLinear, true, true);
      else ENS_STEP(kLawLinear, false, true);
    }
  } else {
    if (g.law == kLawReference) {   // plane walls only
      if (cap) ENS_STEP(kLawReference, true, false);
      else ENS_STEP(kLawReference, false, false);
    } else if (g.law == kLawHertz) {
      if (cap) ENS_STEP(kLawHertz, true, false);
      else ENS_STEP(kLawHertz, false, false);
    } else {
      if (cap) ENS_STEP(kLawLinear, true, false);
      else ENS_STEP(kLawLinear, false, false);
    }
  }
#undef ENS_STEP_MIX
#undef ENS_STEP_ROT
#undef ENS_STEP
#undef ENS_ARGS
}

void ens_launch_step_record(const EnsGeom& g, const EnsBufs& b, int cur, int n, StepCtl* ctl,
                            StepLink link, const EnsTape& tape, int block, cudaStream_t st) {
  const int bs = block >= 64 && block <= kMaxStepBlock && block % 32 == 0 ? block : kThreads;
  const int gs = (n + bs - 1) / bs;
  // reverse mode accepts plane walls only (blaze_ens_adj_create)
  k_ens_step_rec<<<gs, bs, 0, st>>>(g, b, b.S[cur], b.S[2], b.S[cur ^ 1], n, ctl, link, tape);
}

int ens_persist_grid(const EnsGeom& g, int block, int n) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  cudaError_t err;
  if (g.law == kLawReference)
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_persist<kLawReference, false>, block, 0);
  else if (g.curved)
    err = g.law == kLawHertz
              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_persist<kLawHertz, true>, block, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_persist<kLawLinear, true>, block, 0);
  else
    err = g.law == kLawHertz
              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_persist<kLawHertz, false>, block, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_persist<kLawLinear, false>, block, 0);
  if (err != cudaSuccess || per_sm < 1) return 0;
  const int need = (n + block - 1) / block;
  return std::max(1, std::min(need, per_sm * sms));
}

cudaError_t ens_launch_persist(const EnsGeom& g, const EnsBufs& b, int home, int n, StepCtl* ctl,
                               const int* rebuilt, const EnsPersist& p, int block, int grid,
                               bool coop, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = coop ? 1 : 0;
  const StateBuf sh = b.S[home], so = b.S[home ^ 1], ss = b.S[2];
  if (g.law == kLawReference)
    return cudaLaunchKernelEx(&cfg, k_ens_persist<kLawReference, false>, g, b, sh, so, ss, n, ctl, rebuilt, p);
  if (g.curved) {
    if (g.law == kLawHertz)
      return cudaLaunchKernelEx(&cfg, k_ens_persist<kLawHertz, true>, g, b, sh, so, ss, n, ctl, rebuilt, p);
    return cudaLaunchKernelEx(&cfg, k_ens_persist<kLawLinear, true>, g, b, sh, so, ss, n, ctl, rebuilt, p);
  }
  if (g.law == kLawHertz)
    return cudaLaunchKernelEx(&cfg, k_ens_persist<kLawHertz, false>, g, b, sh, so, ss, n, ctl, rebuilt, p);
  return cudaLaunchKernelEx(&cfg, k_ens_persist<kLawLinear, false>, g, b, sh, so, ss, n, ctl, rebuilt, p);
}

void ens_launch_rot_tick(const EnsGeom& g, int nsys, cudaStream_t st) {
  k_ens_rot_tick<<<(nsys + kThreads - 1) / kThreads, kThreads, 0, st>>>(g.sys, g.rot, nsys);
}

void ens_launch_barrier_check(unsigned int* bar, StepCtl* ctl, cudaStream_t st) {
  k_barrier_check<<<2, 64, 0, st>>>(bar, ctl);
}

void ens_launch_persist_gate(StepCtl* ctl, const EnsPersist& p, int* rb,
                             cudaGraphConditionalHandle if_h, cudaStream_t st) {
  k_ens_persist_gate<<<1, 1, 0, st>>>(ctl, p, rb, if_h);
}

void ens_launch_persist_init(const EnsPersist& p, int steps, cudaStream_t st) {
  k_ens_persist_init<<<1, 1, 0, st>>>(p, steps);
}

void ens_launch_pack(const float* pos3, const float* rad, const float* vel3, const float* avel3,
                     const int* sys_of, const EnsBufs& b, int cur, int* pid_dst, int n,
                     int* flags, cudaStream_t st) {
  k_ens_pack<<<nblk(n), kThreads, 0, st>>>(pos3, rad, vel3, avel3, sys_of, b.S[cur], pid_dst,
                                           b.L[0], b.L[1], n, flags);
}

void ens_launch_unpack(const EnsBufs& b, int cur, int n, const int* pid_src, float* pos3,
                       float* rad, float* vel3, float* avel3, int* sys, int* pid,
                       cudaStream_t st) {
  k_ens_unpack<<<nblk(n), kThreads, 0, st>>>(b.S[cur], pid_src, n, pos3, rad, vel3, avel3, sys,
                                             pid);
}

}  // namespace blaze
