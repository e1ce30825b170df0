// mix_kernels.cu -- the ensemble's polyhedron kernels (see mix_kernels.cuh).
#include "mix_kernels.cuh"

#include <climits>

namespace blaze {
namespace {

constexpr int kThreads = 256;
constexpr int kMixWarps = 4;      // warps (polyhedra) per block of the step
constexpr int kMixHits = 32;      // touching triangles kept per polyhedron and step

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

// --------------------------------------------------------------- marking
__global__ void __launch_bounds__(kThreads)
k_mix_mark(StateBuf s, MixBufs m, const int* __restrict__ caller_index,
           const float4* __restrict__ quat) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.npoly) return;
  const int i = caller_index[p];
  const float rb = m.shapes[m.shape_of[p]].rb;
  float4 x = s.pos[i];
  x.w = -rb;
  s.pos[i] = x;
  float4 w = s.angv[i];
  w.w = __int_as_float(p);
  s.angv[i] = w;
  m.quat[p] = quat[p];
  m.pat[p] = i;
  m.ppath[p] = 0.0f;
  m.wn[p] = 0;
  for (int c = 0; c < 2; ++c) {
    m.L[c].cnt[p] = 0;
    m.L[c].mlo[p] = 0;
    m.L[c].mhi[p] = 0;
  }
}

// -------------------------------------------------------------- geometry
// One thread per (polyhedron, vertex or face).
__global__ void __launch_bounds__(kThreads)
k_mix_geom(MixBufs m) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = t / (kMixMaxV + kMixMaxF), item = t % (kMixMaxV + kMixMaxF);
  if (p >= m.npoly) return;
  const int s = m.shape_of[p];
  const MixShapeDev& SH = m.shapes[s];
  double R[9];
  mix_rotation(m.quat[p], R);
  if (item < kMixMaxV) {
    if (item >= SH.nv) return;
    const float4 b = m.bv[(size_t)s * kMixMaxV + item];
    const double3 v = mat_vec(R, dv(b.x, b.y, b.z));
    m.gv[(size_t)p * kMixMaxV + item] = make_double4(v.x, v.y, v.z, 0.0);
  } else {
    const int f = item - kMixMaxV;
    if (f >= SH.nf) return;
    const double3 n = mat_vec(R, dxyz(m.bn[(size_t)s * kMixMaxF + f]));
    const float4 b = m.bv[(size_t)s * kMixMaxV + m.faces[(size_t)s * kMixMaxF + f].x];
    const double3 v = mat_vec(R, dv(b.x, b.y, b.z));
    m.gf[(size_t)p * kMixMaxF + f] = make_double4(n.x, n.y, n.z, ddot(n, v));
  }
}

// -------------------------------------------------------------- the list
// Pairs with |xi - xj|^2 < (ri + rj + skin)^2 (bounding radii) from the 27
// surrounding cells, in the sphere list's order (z, y, x; j ascending); the
// history of an old slot moves to the new slot of the same partner pid.  A
// warp per polyhedron: the lanes take consecutive candidates of a cell and
// a ballot hands out the slots in candidate order.
__global__ void __launch_bounds__(kThreads)
k_mix_plist(EnsGeom g, EnsBufs b, MixBufs m, const float4* __restrict__ pos,
            const float4* __restrict__ vel, const uint32_t* __restrict__ cstart,
            const uint32_t* __restrict__ cend, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int lane = threadIdx.x & 31;
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= m.npoly) return;
  const int e = ctl->epoch & 1;
  const MixList Lo = m.L[e], Ln = m.L[e ^ 1];
  const int* pid_old = b.pid[e];
  const int* pid_new = b.pid[e ^ 1];
  const size_t P = (size_t)m.npoly;
  const int i = m.pat[p];
  const float4 pa4 = pos[i];
  const float3 pa = xyz(pa4);
  const float ra = fabsf(pa4.w);
  const uint32_t sys = __float_as_uint(vel[i].w) & kSysMask;
  const EnsSysDev& S = g.sys[sys];
  const int3 c = ens_cell(S, pa);
  const uint32_t cnt_o = Lo.cnt[p];
  const unsigned long long mask_o =
      (unsigned long long)Lo.mlo[p] | ((unsigned long long)Lo.mhi[p] << 32);
  uint32_t cnt = 0, st = 0;
  unsigned long long mask = 0;   // lane-local bits, merged at the end
  if (ens_in(S, c)) {
    const int x0 = c.x > 0 ? c.x - 1 : 0, x1 = c.x < S.nc.x - 1 ? c.x + 1 : c.x;
    const int y0 = c.y > 0 ? c.y - 1 : 0, y1 = c.y < S.nc.y - 1 ? c.y + 1 : c.y;
    const int z0 = c.z > 0 ? c.z - 1 : 0, z1 = c.z < S.nc.z - 1 ? c.z + 1 : c.z;
    for (int z = z0; z <= z1; ++z)
      for (int y = y0; y <= y1; ++y) {
        const uint32_t row = S.cell_off + (uint32_t)(S.nc.x * (y + S.nc.y * z));
        for (int x = x0; x <= x1; ++x) {
          const uint32_t h = row + (uint32_t)x;
          const uint32_t s0 = __ldg(cstart + h);
          if (s0 == 0xffffffffu) continue;
          const uint32_t eo = __ldg(cend + h);
          for (uint32_t j0 = s0; j0 < eo; j0 += 32) {
            const uint32_t j = j0 + (uint32_t)lane;
            bool hit = false;
            if (j < eo && (int)j != i) {
              const float4 pb = __ldg(pos + j);
              const float3 rel = pa - xyz(pb);
              const float lim = (ra + fabsf(pb.w)) + g.skin;
              hit = dot3(rel, rel) < lim * lim;
            }
            const uint32_t hb = __ballot_sync(0xffffffffu, hit);
            if (hit) {
              const uint32_t k = cnt + (uint32_t)__popc(hb & ((1u << lane) - 1u));
              if (k < (uint32_t)kMixSlots) {
                Ln.idx[(size_t)k * P + p] = j;
                Ln.sep[(size_t)k * P + p] = -1;
                unsigned long long mo = mask_o;
                if (mo) {
                  const int pj = pid_new[j];
                  while (mo) {
                    const int ko = __ffsll((long long)mo) - 1;
                    mo &= mo - 1ull;
                    if ((uint32_t)ko >= cnt_o) break;
                    const size_t so = (size_t)ko * P + p;
                    if (pid_old[Lo.idx[so]] == pj) {
                      const size_t sn = (size_t)k * P + p;
                      Ln.hx[sn] = Lo.hx[so];
                      Ln.hy[sn] = Lo.hy[so];
                      Ln.hz[sn] = Lo.hz[so];
                      mask |= 1ull << k;
                      break;
                    }
                  }
                }
              } else {
                st |= kStatusListOverflow;
              }
            }
            cnt += (uint32_t)__popc(hb);
          }
        }
      }
  } else {
    st |= kStatusOutOfGrid;
  }
  // the lanes' history bits together
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mask |= __shfl_xor_sync(0xffffffffu, mask, o);
  st = __reduce_or_sync(0xffffffffu, st);
  if (lane == 0) {
    Ln.cnt[p] = cnt < (uint32_t)kMixSlots ? cnt : (uint32_t)kMixSlots;
    Ln.mlo[p] = (uint32_t)mask;
    Ln.mhi[p] = (uint32_t)(mask >> 32);
    if (st) atomicOr(&ctl->status, st);
  }
}

// The twin of every sphere slot that holds a polyhedron: the polyhedron's
// slot that holds the sphere (new lists, before the epoch turns).
__global__ void __launch_bounds__(kThreads)
k_mix_twins(EnsBufs b, MixBufs m, const float4* __restrict__ pos,
            const float4* __restrict__ angv, int n, StepCtl* ctl, const int* gate) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (pos[i].w < 0.0f) return;
  const int e = ctl->epoch & 1;
  const EnsList Ln = b.L[e ^ 1];
  const MixList Pn = m.L[e ^ 1];
  const size_t stride = (size_t)b.stride, P = (size_t)m.npoly;
  const uint32_t cnt = Ln.cnt[i];
  uint32_t st = 0;
  for (uint32_t k = 0; k < cnt; ++k) {
    const size_t sk = (size_t)k * stride + i;
    const uint32_t j = Ln.idx[sk];
    if (!(pos[j].w < 0.0f)) continue;
    const int q = __float_as_int(angv[j].w);
    const uint32_t c = Pn.cnt[q];
    uint32_t tw = 0xffu;
    for (uint32_t kk = 0; kk < c; ++kk)
      if (Pn.idx[(size_t)kk * P + q] == (uint32_t)i) { tw = kk; break; }
    if (tw == 0xffu) st |= kStatusListOverflow;
    m.twin[sk] = (uint8_t)tw;
  }
  if (st) atomicOr(&ctl->status, st);
}

// -------------------------------------------------------------- the step
// (value, index) maximum over the warp, the lowest index on ties: the
// serial loop's first maximum.
__device__ __forceinline__ void warp_argmax(double& s, int& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
    if (s2 > s || (s2 == s && i2 < i)) {
      s = s2;
      i = i2;
    }
  }
}

struct HullRef {
  const double4* V;
  const double4* F;
  const uchar4* E;
  int nv, nf, ne;
};

// The edge pair x = ea * B.ne + eb of hulls A and B (B's centre at d).
__device__ __forceinline__ double pair_edge_sep(double3 d, const HullRef& A, const HullRef& B,
                                                int x) {
  const uchar4 ea = A.E[x / B.ne], eb = B.E[x % B.ne];
  return edge_sep(dxyz(A.F[ea.z]), dxyz(A.F[ea.w]), dxyz(B.F[eb.z]), dxyz(B.F[eb.w]),
                  dxyz(A.V[ea.x]), dxyz(A.V[ea.y]), dadd(d, dxyz(B.V[eb.x])),
                  dadd(d, dxyz(B.V[eb.y])));
}

// Whether the axis `code` (MixList::sep) separates hulls A and B.
__device__ __forceinline__ bool axis_separates(int code, double3 d, const HullRef& A,
                                               const HullRef& B) {
  const int kind = code >> 16, x = code & 0xffff;
  if (kind == 0) return face_sep(A.F[x], d, B.V, B.nv) > 0.0;
  if (kind == 1) return face_sep(B.F[x], dneg(d), A.V, A.nv) > 0.0;
  return pair_edge_sep(d, A, B, x) > 0.0;
}

// The separating-axis queries of hulls A and B (B's centre at d from A's),
// shared by the warp: false when an axis separates them (its code in sep).
__device__ bool hull_hull_warp(int lane, double3 d, const HullRef& A, const HullRef& B,
                               SatPick& q, int& sep) {
  double s = -1e300;
  int k = INT_MAX;
  for (int f = lane; f < A.nf; f += 32) {
    const double t = face_sep(A.F[f], d, B.V, B.nv);
    if (t > s) { s = t; k = f; }
  }
  warp_argmax(s, k);
  if (s > 0.0) {
    sep = k;
    return false;
  }
  q.sA = s;
  q.fA = k;
  const double3 md = dneg(d);
  s = -1e300;
  k = INT_MAX;
  for (int f = lane; f < B.nf; f += 32) {
    const double t = face_sep(B.F[f], md, A.V, A.nv);
    if (t > s) { s = t; k = f; }
  }
  warp_argmax(s, k);
  if (s > 0.0) {
    sep = (1 << 16) | k;
    return false;
  }
  q.sB = s;
  q.fB = k;
  s = kNoAxis;
  k = INT_MAX;
  const int tot = A.ne * B.ne;
  for (int x = lane; x < tot; x += 32) {
    const double t = pair_edge_sep(d, A, B, x);
    if (t > s) { s = t; k = x; }
  }
  warp_argmax(s, k);
  if (s > 0.0) {
    sep = (2 << 16) | k;
    return false;
  }
  q.sE = s;
  q.eE = k;
  return true;
}

// warp minimum / maximum of a double (exact: no rounding)
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// hull_tri with its queries shared by the warp: the polyhedron's faces, its
// extent along the triangle's normal and the 3 ne edge-pair axes split over
// the lanes; the maxima taken with the lowest index on ties, which is the
// serial loop's answer; the contact from the same hull_tri_finish.
__device__ bool hull_tri_warp(int lane, const HullRef& D, const double3* T, double3 nt, MixHit& h,
                              double3& nd, int& kind) {
  double sP = -1e300;
  int fP = INT_MAX;
  for (int f = lane; f < D.nf; f += 32) {
    const double s = tri_face_sep(D.F[f], T);
    if (s > sP) { sP = s; fP = f; }
  }
  warp_argmax(sP, fP);
  if (sP > 0.0) return false;
  double lo = 1e300, hi = -1e300;
  for (int k = lane; k < D.nv; k += 32) {
    const double t = ddot(nt, dxyz(D.V[k]));
    lo = fmin(lo, t);
    hi = fmax(hi, t);
  }
  lo = warp_min(lo);
  hi = warp_max(hi);
  bool tplus;
  const double sT = tri_plane_sep(nt, T, lo, hi, tplus);
  if (sT > 0.0) return false;
  double sE = -1e300;
  int eE = INT_MAX;
  bool sep = false;
  for (int x = lane; x < 3 * D.ne; x += 32) {
    bool pl;
    const double s = tri_edge_sep(D.V, D.E, D.nv, T, x, pl);
    if (s == kNoAxis) continue;
    if (s > 0.0) sep = true;
    if (s > sE) { sE = s; eE = x; }
  }
  if (__any_sync(0xffffffffu, sep)) return false;
  warp_argmax(sE, eE);
  bool eplus = true;
  if (eE == INT_MAX) {
    eE = -1;
  } else {
    tri_edge_sep(D.V, D.E, D.nv, T, eE, eplus);
  }
  return hull_tri_finish(D.V, D.F, D.E, D.nv, T, nt, sT, tplus, sP, fP, sE, eE, eplus, h, nd,
                         kind);
}

struct MixSmem {
  float4 f[kMixSlots];      // per slot: force and torque on this polyhedron
  float4 t[kMixSlots];
  double4 v[kMixMaxV];      // geometry in the drum's frame (a turning drum)
  double4 fn[kMixMaxF];
  double3 nd[kMixHits];     // touching triangles: unrounded normal, contact, id
  MixHit hit[kMixHits];
  int hid[kMixHits];
  int hkind[kMixHits];      // 0: the triangle's face; 1, 2: a face of the polyhedron, an edge pair
  float4 oh[kMixWallSlots]; // the polyhedron's wall histories before the step
};

__device__ __forceinline__ float3 mat_vec_f(const float* R, float3 v) {
  return f3((R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
            (R[6] * v.x + R[7] * v.y) + R[8] * v.z);
}
__device__ __forceinline__ float3 mat_tvec_f(const float* R, float3 v) {
  return f3((R[0] * v.x + R[3] * v.y) + R[6] * v.z, (R[1] * v.x + R[4] * v.y) + R[7] * v.z,
            (R[2] * v.x + R[5] * v.y) + R[8] * v.z);
}

// One warp per polyhedron.  The polyhedron's own force is summed by lane 0
// in slot order, then the walls (planes in order, then the kept triangles
// in ascending id), as the restatement sums.
template <bool kCapture, bool kRot>
__global__ void __launch_bounds__(32 * kMixWarps, 4)
k_mix_poly_step(EnsGeom g, EnsBufs b, MixBufs m, StateBuf in_plain, StateBuf in_sorted,
                StateBuf out, StepCtl* ctl, StepLink link, EnsCapture cap) {
  __shared__ MixSmem smem[kMixWarps];
  const int lane = threadIdx.x & 31;
  MixSmem& sm = smem[threadIdx.x >> 5];
  const int p = blockIdx.x * kMixWarps + (int)(threadIdx.x >> 5);
  if (p >= m.npoly) return;
  const bool rebuilt = *link.rebuilt != 0;
  const StateBuf in = rebuilt ? in_sorted : in_plain;
  const int e = ctl->epoch & 1;
  const MixList L = m.L[e];
  const size_t P = (size_t)m.npoly;
  const int i = m.pat[p];
  const float4 pa4 = in.pos[i], va4 = in.vel[i], wa4 = in.angv[i];
  const float3 xa = xyz(pa4), va = xyz(va4), wa = xyz(wa4);
  const uint32_t sys = __float_as_uint(va4.w) & kSysMask;
  const EnsSysDev& S = g.sys[sys];
  const int shp = m.shape_of[p];
  const MixShapeDev& SH = m.shapes[shp];
  const float mass = SH.mass, rb = SH.rb;
  HullRef A;
  A.V = m.gv + (size_t)p * kMixMaxV;
  A.F = m.gf + (size_t)p * kMixMaxF;
  A.E = m.edges + (size_t)shp * kMixMaxE;
  A.nv = SH.nv;
  A.nf = SH.nf;
  A.ne = SH.ne;
  const uchar4* faces = m.faces + (size_t)shp * kMixMaxF;
  const float dt = g.dt;
  const uint32_t cnt = L.cnt[p];
  const uint32_t mlo = L.mlo[p], mhi = L.mhi[p];
  uint32_t st = 0;

  // sphere neighbours: a slot per lane
  uint32_t touch[2], polys[2];
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const uint32_t k = (uint32_t)lane + 32u * (uint32_t)half;
    bool is_poly = false, touched = false;
    if (k < cnt) {
      const size_t sk = (size_t)k * P + p;
      const uint32_t j = L.idx[sk];
      const float4 pb4 = in.pos[j];
      if (pb4.w < 0.0f) {
        is_poly = true;
      } else {
        // the pair is evaluated here only: the sphere's step reads the force
        // and torque on it from sf / st
        const float3 rel = xyz(pb4) - xa;
        const float sr = pb4.w + rb;
        const float d2 = dot3(rel, rel);
        MixHit h;
        float4 sfo = make_float4(0.0f, 0.0f, 0.0f, 0.0f), sto = sfo;
        if (d2 < sr * sr && sqrtf(d2) > 0.0f &&
            sphere_hull(xyz(pb4), pb4.w, xa, A.V, A.F, faces, A.nf, h)) {
          const float4 vb4 = in.vel[j], wb4 = in.angv[j];
          float3 xi = f3(0.0f, 0.0f, 0.0f);
          if ((((half ? mhi : mlo) >> lane) & 1u) != 0u) xi = f3(L.hx[sk], L.hy[sk], L.hz[sk]);
          float3 F, Ts, Tp;
          mix_pair_law(S, h, sphere_mass(S, pb4.w), xyz(vb4), xyz(wb4), mass, va, wa, dt, xi, F,
                       Ts, Tp);
          L.hx[sk] = xi.x;
          L.hy[sk] = xi.y;
          L.hz[sk] = xi.z;
          sm.f[k] = make_float4(-F.x, -F.y, -F.z, 0.0f);
          sm.t[k] = make_float4(Tp.x, Tp.y, Tp.z, 0.0f);
          sfo = make_float4(F.x, F.y, F.z, 1.0f);
          sto = make_float4(Ts.x, Ts.y, Ts.z, 0.0f);
          touched = true;
        }
        m.sf[sk] = sfo;
        m.st[sk] = sto;
      }
    }
    touch[half] = __ballot_sync(0xffffffffu, touched);
    polys[half] = __ballot_sync(0xffffffffu, is_poly);
  }

  // polyhedron neighbours: the warp on one pair at a time
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    uint32_t pm = polys[half];
    while (pm) {
      const int bit = __ffs(pm) - 1;
      pm &= pm - 1u;
      const uint32_t k = (uint32_t)bit + 32u * (uint32_t)half;
      const size_t sk = (size_t)k * P + p;
      const uint32_t j = L.idx[sk];
      const float4 pb4 = in.pos[j], vb4 = in.vel[j], wb4 = in.angv[j];
      const int q = __float_as_int(wb4.w);
      const int sq = m.shape_of[q];
      const bool selfA = p < q;
      const float3 xA = selfA ? xa : xyz(pb4), xB = selfA ? xyz(pb4) : xa;
      const float rA = selfA ? rb : -pb4.w, rB = selfA ? -pb4.w : rb;
      const float3 rel = xB - xA;
      const float sr = rA + rB;
      if (!(dot3(rel, rel) < sr * sr)) continue;
      HullRef Bq;
      Bq.V = m.gv + (size_t)q * kMixMaxV;
      Bq.F = m.gf + (size_t)q * kMixMaxF;
      Bq.E = m.edges + (size_t)sq * kMixMaxE;
      Bq.nv = m.shapes[sq].nv;
      Bq.nf = m.shapes[sq].nf;
      Bq.ne = m.shapes[sq].ne;
      const HullRef& HA = selfA ? A : Bq;
      const HullRef& HB = selfA ? Bq : A;
      const double3 d = dsub(d3(xB), d3(xA));
      const int code = L.sep[sk];
      if (code >= 0 && axis_separates(code, d, HA, HB)) continue;
      SatPick pick;
      int scode;
      if (!hull_hull_warp(lane, d, HA, HB, pick, scode)) {
        if (lane == 0 && scode != code) L.sep[sk] = scode;
        continue;
      }
      MixHit h;
      if (!hull_hull_finish(pick, d, HA.V, HA.F, HA.E, HA.nv, HB.V, HB.F, HB.E, HB.nv, HB.ne, h))
        continue;
      if (lane == 0) {
        float3 xi = f3(0.0f, 0.0f, 0.0f);
        if ((((half ? mhi : mlo) >> bit) & 1u) != 0u) xi = f3(L.hx[sk], L.hy[sk], L.hz[sk]);
        const float mq = m.shapes[sq].mass;
        float3 F, TA, TB;
        if (selfA) mix_pair_law(S, h, mass, va, wa, mq, xyz(vb4), xyz(wb4), dt, xi, F, TA, TB);
        else mix_pair_law(S, h, mq, xyz(vb4), xyz(wb4), mass, va, wa, dt, xi, F, TA, TB);
        L.hx[sk] = xi.x;
        L.hy[sk] = xi.y;
        L.hz[sk] = xi.z;
        sm.f[k] = selfA ? make_float4(F.x, F.y, F.z, 0.0f) : make_float4(-F.x, -F.y, -F.z, 0.0f);
        sm.t[k] = selfA ? make_float4(TA.x, TA.y, TA.z, 0.0f) : make_float4(TB.x, TB.y, TB.z, 0.0f);
      }
      touch[half] |= 1u << bit;
    }
  }

  // triangles: a candidate per lane, in the drum's frame when it turns
  int nhit = 0;
  bool rot = false;
  float rc = 1.0f, rsn = 0.0f;
  if constexpr (kRot) {
    if (S.rot) {
      rot = true;
      const float2 cs = g.rot[sys];
      rc = cs.x;
      rsn = cs.y;
    }
  }
  if (g.tri_off) {
    const float3 pd = rot ? S.rot_o + rot_about(S.rot_a, rc, -rsn, xa - S.rot_o) : xa;
    const int3 c = ens_cell(S, pd);
    if (ens_in(S, c)) {
      const uint32_t hcell = ens_key(S, c);
      const uint32_t o0 = __ldg(g.tri_off + hcell), o1 = __ldg(g.tri_off + hcell + 1);
      if (o1 > o0) {
        HullRef D = A;
        if (rot) {
          const double3 ax = d3(S.rot_a);
          const double cc = (double)rc, ss = -(double)rsn;
          for (int it = lane; it < A.nv + A.nf; it += 32) {
            if (it < A.nv) {
              const double3 v = rot_about_d(ax, cc, ss, dxyz(A.V[it]));
              sm.v[it] = make_double4(v.x, v.y, v.z, 0.0);
            } else {
              const double4 P4 = A.F[it - A.nv];
              const double3 n = rot_about_d(ax, cc, ss, dxyz(P4));
              sm.fn[it - A.nv] = make_double4(n.x, n.y, n.z, P4.w);
            }
          }
          __syncwarp();
          D.V = sm.v;
          D.F = sm.fn;
        }
        // candidates near the polyhedron (a lane each), then the test of
        // each, in ascending order, by the whole warp
        const float lim = rb * 1.001f + 1e-3f;
        for (uint32_t q0 = o0; q0 < o1; q0 += 32) {
          const uint32_t qq = q0 + (uint32_t)lane;
          bool near = false;
          int id = -1;
          if (qq < o1) {
            id = (int)__ldg(g.tri_ids + qq);
            const EnsWallDev& W = g.walls[id];
            int region, feat;
            const float3 cp = closest_on_triangle(pd, W.a, W.b, W.c, region, feat);
            const float3 dd = pd - cp;
            near = dot3(dd, dd) < lim * lim;
          }
          uint32_t nb = __ballot_sync(0xffffffffu, near);
          while (nb) {
            const int src = __ffs(nb) - 1;
            nb &= nb - 1u;
            const int tid = __shfl_sync(0xffffffffu, id, src);
            const EnsWallDev& W = g.walls[tid];
            const double3 o = d3(pd);
            double3 T[3];
            T[0] = dsub(d3(W.a), o);
            T[1] = dsub(d3(W.b), o);
            T[2] = dsub(d3(W.c), o);
            MixHit h;
            double3 nd;
            int kind;
            if (!hull_tri_warp(lane, D, T, W.n64, h, nd, kind)) continue;
            if (lane == 0 && nhit < kMixHits) {
              sm.hit[nhit] = h;
              sm.nd[nhit] = nd;
              sm.hid[nhit] = tid;
              sm.hkind[nhit] = kind;
            }
            ++nhit;
          }
        }
        if (nhit > kMixHits) {
          st |= kStatusListOverflow;
          nhit = kMixHits;
        }
        __syncwarp();
      }
    }
  }

  if (lane == 0) {
    float3 f = f3(0.0f, 0.0f, 0.0f), t = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t tm = touch[half];
      while (tm) {
        const int k = __ffs(tm) - 1 + 32 * half;
        tm &= tm - 1u;
        f = f + xyz(sm.f[k]);
        t = t + xyz(sm.t[k]);
      }
    }
    if (touch[0] != mlo) L.mlo[p] = touch[0];
    if (touch[1] != mhi) L.mhi[p] = touch[1];

    // walls: the old history slots (by wall id), new ones written in
    // processing order over them
    float4* wh = m.wh + (size_t)p * kMixWallSlots;
    const int nw_o = m.wn[p];
    float4* oh = sm.oh;
    for (int qs = 0; qs < nw_o; ++qs) oh[qs] = wh[qs];
    int nw = 0;
    auto wall = [&](int id, const MixHit& h, bool moving) {
      float3 xi = f3(0.0f, 0.0f, 0.0f);
      for (int qs = 0; qs < nw_o; ++qs)
        if (__float_as_int(oh[qs].w) == id) xi = f3(oh[qs].x, oh[qs].y, oh[qs].z);
      const float3 vw = moving ? cross3(S.rot_a, (xa + h.ca) - S.rot_o) * S.rot_w
                               : f3(0.0f, 0.0f, 0.0f);
      float3 F, T;
      mix_wall_law(S, h, mass, va, wa, vw, dt, xi, F, T);
      f = f + F;
      t = t + T;
      if (nw < kMixWallSlots) {
        wh[nw] = make_float4(xi.x, xi.y, xi.z, __int_as_float(id));
        ++nw;
      } else {
        st |= kStatusListOverflow;
      }
    };
    for (int w = S.wall0; w < S.wall0 + S.nwall; ++w) {
      const EnsWallDev& W = g.walls[w];
      MixHit h;
      if (W.kind == kWallPlane && hull_plane(W.a, W.r, xa, A.V, A.nv, h))
        wall(w, h, rot && W.turning);
    }
    // contacts with a triangle's face all count, those of one plane once
    // (the deepest); without one, only the deepest other contact does (a
    // polyhedron over the shared edge of two triangles of a flat or concave
    // region touches it once)
    bool anyface = false;
    int best = -1;
    for (int a = 0; a < nhit; ++a) {
      if (sm.hkind[a] == 0) anyface = true;
      else if (best < 0 || sm.hit[a].delta > sm.hit[best].delta) best = a;
    }
    for (int a = 0; a < nhit; ++a) {
      bool keep = anyface ? sm.hkind[a] == 0 : a == best;
      for (int c2 = 0; c2 < nhit && keep && anyface; ++c2) {
        if (c2 == a || sm.hkind[c2] != 0 || !(ddot(sm.nd[a], sm.nd[c2]) > kMixCoplanar)) continue;
        const float da = sm.hit[a].delta, dc = sm.hit[c2].delta;
        if (dc > da || (dc == da && sm.hid[c2] < sm.hid[a])) keep = false;
      }
      if (!keep) continue;
      MixHit h = sm.hit[a];
      if (rot) {
        h.n = rot_about(S.rot_a, rc, rsn, h.n);
        h.ca = rot_about(S.rot_a, rc, rsn, h.ca);
      }
      wall(sm.hid[a], h, rot);
    }
    m.wn[p] = nw;

    // symplectic Euler: translation; rotation by Euler's equations in the
    // body frame, then the quaternion
    const float inv_m = 1.0f / mass;
    const float3 acc = f * inv_m + S.gravity;
    const float3 v = va + acc * dt;
    const float3 x = xa + v * dt;
    const float4 q4 = m.quat[p];
    const float qw = q4.x, qx = q4.y, qy = q4.z, qz = q4.w;
    float R[9];
    {
      const float s = 2.0f / (((qw * qw + qx * qx) + qy * qy) + qz * qz);
      R[0] = 1.0f - s * (qy * qy + qz * qz);
      R[1] = s * (qx * qy - qw * qz);
      R[2] = s * (qx * qz + qw * qy);
      R[3] = s * (qx * qy + qw * qz);
      R[4] = 1.0f - s * (qx * qx + qz * qz);
      R[5] = s * (qy * qz - qw * qx);
      R[6] = s * (qx * qz - qw * qy);
      R[7] = s * (qy * qz + qw * qx);
      R[8] = 1.0f - s * (qx * qx + qy * qy);
    }
    const float3 tb = mat_tvec_f(R, t), wb = mat_tvec_f(R, wa);
    const float3 lb = mat_vec_f(SH.inertia, wb);
    const float3 dwb = mat_vec_f(SH.iinv, tb - cross3(wb, lb));
    const float3 w = mat_vec_f(R, wb + dwb * dt);
    const float hdt = 0.5f * dt;
    const float nw_ = -((w.x * qx + w.y * qy) + w.z * qz);
    const float3 nv_ = f3(qw * w.x, qw * w.y, qw * w.z) + cross3(w, f3(qx, qy, qz));
    float q2w = qw + hdt * nw_, q2x = qx + hdt * nv_.x, q2y = qy + hdt * nv_.y,
          q2z = qz + hdt * nv_.z;
    const float qi = 1.0f / sqrtf(((q2w * q2w + q2x * q2x) + q2y * q2y) + q2z * q2z);
    q2w = q2w * qi;
    q2x = q2x * qi;
    q2y = q2y * qi;
    q2z = q2z * qi;
    const float path = m.ppath[p] + len3(v) * dt;
    out.pos[i] = make_float4(x.x, x.y, x.z, -rb);
    out.vel[i] = make_float4(v.x, v.y, v.z, __uint_as_float(sys));
    out.angv[i] = make_float4(w.x, w.y, w.z, __int_as_float(p));
    m.quat[p] = make_float4(q2w, q2x, q2y, q2z);
    m.ppath[p] = path;
    if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z))) st |= kStatusNonFinite;
    if (kCapture) {
      cap.f[i] = make_float4(f.x, f.y, f.z, 0.0f);
      cap.t[i] = make_float4(t.x, t.y, t.z, 0.0f);
    }
    if (path > 0.5f * g.skin) {
      if (link.has_next_h) cudaGraphSetConditional(link.next_h, 1u);
      else atomicExch(&ctl->rebuild_req, 1);
    }
  }
  st = __reduce_or_sync(0xffffffffu, st);
  if (lane == 0 && st) atomicOr(&ctl->status, st);
}

}  // namespace

void mix_launch_mark(const EnsBufs& b, int cur, const MixBufs& m, const int* caller_index,
                     const float4* quat, cudaStream_t st) {
  if (m.npoly <= 0) return;
  k_mix_mark<<<nblk(m.npoly), kThreads, 0, st>>>(b.S[cur], m, caller_index, quat);
}

void mix_launch_geom(const MixBufs& m, cudaStream_t st) {
  if (m.npoly <= 0) return;
  k_mix_geom<<<nblk(m.npoly * (kMixMaxV + kMixMaxF)), kThreads, 0, st>>>(m);
}

void mix_launch_plist(const EnsGeom& g, const EnsBufs& b, const MixBufs& m,
                      const uint32_t* cstart, const uint32_t* cend, StepCtl* ctl,
                      const int* gate, cudaStream_t st) {
  if (m.npoly <= 0) return;
  k_mix_plist<<<nblk(32 * m.npoly), kThreads, 0, st>>>(g, b, m, b.S[2].pos, b.S[2].vel, cstart,
                                                       cend, ctl, gate);
}

void mix_launch_twins(const EnsBufs& b, const MixBufs& m, int n, StepCtl* ctl, const int* gate,
                      cudaStream_t st) {
  if (m.npoly <= 0) return;
  k_mix_twins<<<nblk(n), kThreads, 0, st>>>(b, m, b.S[2].pos, b.S[2].angv, n, ctl, gate);
}

void mix_launch_poly_step(const EnsGeom& g, const EnsBufs& b, const MixBufs& m, int cur,
                          StepCtl* ctl, StepLink link, const EnsCapture* cap, cudaStream_t st) {
  if (m.npoly <= 0) return;
  const EnsCapture c = cap ? *cap : EnsCapture{nullptr, nullptr};
  const int gs = (m.npoly + kMixWarps - 1) / kMixWarps;
#define MIX_ARGS g, b, m, b.S[cur], b.S[2], b.S[cur ^ 1], ctl, link, c
  if (g.any_rot) {
    if (cap) k_mix_poly_step<true, true><<<gs, 32 * kMixWarps, 0, st>>>(MIX_ARGS);
    else k_mix_poly_step<false, true><<<gs, 32 * kMixWarps, 0, st>>>(MIX_ARGS);
  } else {
    if (cap) k_mix_poly_step<true, false><<<gs, 32 * kMixWarps, 0, st>>>(MIX_ARGS);
    else k_mix_poly_step<false, false><<<gs, 32 * kMixWarps, 0, st>>>(MIX_ARGS);
  }
#undef MIX_ARGS
}

}  // namespace blaze
