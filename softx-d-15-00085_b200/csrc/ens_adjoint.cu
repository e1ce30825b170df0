// ens_adjoint.cu -- reverse-mode kernels of the ensemble step (see
// ens_adjoint.cuh).  The contact-law reverse below follows the forward in
// ens_kernels.cu (contact_law, linear law) statement by statement, in
// reverse order.
#include "ens_adjoint.cuh"

namespace blaze {
namespace {

constexpr int kThreads = 128;

struct LawBar { float kn, kt, b2, mu; };
struct SBar { float3 x, v, w; };

__device__ __forceinline__ float3 xyz4(float4 a) { return f3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 w4(float3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }

// Cotangents of contact_law's inputs (n, delta, vrel, vct, xi) and of the
// law constants for cotangents Fb, Tb (force, torque on a) and Xb (history
// after the step).
__device__ void contact_vjp(const EnsSysDev& S, float mu, float3 n, float delta, float ms,
                            float3 vrel, float3 vct, float arm, float3 x, float dt, float3 Fb,
                            float3 Tb, float3 Xb, float3& nb, float& deltab, float3& vrelb,
                            float3& vctb, float3& xb, LawBar& th) {
  const float kn = S.kn, kt = S.kt;
  const float sqn = sqrtf(ms * kn), sqt = sqrtf(ms * kt);
  const float cn = S.beta2 * sqn, ct = S.beta2 * sqt;
  const float vn = dot3(vrel, n);
  const float fn = kn * delta - cn * vn;
  const float fc = fn > 0.0f ? fn : 0.0f;
  const float p = dot3(vct, n);
  const float3 vt = vct - p * n;
  const float xn = dot3(x, n);
  const bool rot = xn != 0.0f;
  float m0 = 0.0f, m1 = 0.0f, g = 1.0f;
  float3 x1 = x;
  if (rot) {
    m0 = dot3(x, x);
    x1 = x - xn * n;
    m1 = dot3(x1, x1);
    if (m1 > 0.0f) g = sqrtf(m0 / m1);
  }
  const float3 x2 = (rot && m1 > 0.0f) ? x1 * g : x1;
  const float3 x3 = x2 + vt * dt;
  const float3 ft = x3 * (-kt) - vt * ct;
  const float cap = mu * fc;
  const float f2 = dot3(ft, ft);
  const bool slip = f2 > cap * cap;
  float fmag = 0.0f, s = 1.0f;
  float3 ftp = ft;
  if (slip) {
    fmag = sqrtf(f2);
    s = cap / fmag;
    ftp = ft * s;
  }
  const float3 F = n * fn + ftp;
  // reverse
  float3 vtb = f3(0.0f, 0.0f, 0.0f), ftb, x3b;
  float fcb = 0.0f, ctb = 0.0f, ktb = 0.0f, knb = 0.0f, cnb = 0.0f, mub = 0.0f;
  xb = f3(0.0f, 0.0f, 0.0f);
  const float3 u = n * (-arm);                 // T = u x F
  nb = cross3(F, Tb) * (-arm);
  const float3 Ft = Fb + cross3(Tb, u);
  float fnb = dot3(Ft, n);                     // F = n fn + ftp
  nb = nb + Ft * fn;
  float3 ftpb = Ft;
  if (slip) {
    const float ik = -1.0f / kt;               // x4 = (ftp + vt ct)(-1/kt)
    const float3 A = ftp + vt * ct;
    ftpb = ftpb + Xb * ik;
    vtb = vtb + Xb * (ik * ct);
    ctb += dot3(vt, Xb) * ik;
    ktb += dot3(A, Xb) / (kt * kt);
    ftb = ftpb * s;                            // ftp = ft s
    const float sb = dot3(ft, ftpb);
    const float capb = sb / fmag;              // s = cap / |ft|
    const float fmagb = -sb * cap / (fmag * fmag);
    ftb = ftb + ft * (fmagb / fmag);
    mub += capb * fc;
    fcb += capb * mu;
    x3b = f3(0.0f, 0.0f, 0.0f);
  } else {
    ftb = ftpb;
    x3b = Xb;
  }
  x3b = x3b + ftb * (-kt);                     // ft = x3 (-kt) - vt ct
  ktb -= dot3(x3, ftb);
  ctb -= dot3(vt, ftb);
  vtb = vtb + ftb * (-ct);
  const float3 x2b = x3b;                      // x3 = x2 + vt dt
  vtb = vtb + x3b * dt;
  if (rot) {
    float3 x1b = x2b;
    if (m1 > 0.0f) {
      x1b = x2b * g;                           // x2 = x1 sqrt(m0 / m1)
      const float gb = dot3(x1, x2b);
      const float m0b = gb * g / (2.0f * m0);
      const float m1b = -gb * g / (2.0f * m1);
      x1b = x1b + x1 * (2.0f * m1b);
      xb = xb + x * (2.0f * m0b);
    }
    xb = xb + x1b;                             // x1 = x - xn n
    const float xnb = -dot3(n, x1b);
    nb = nb + x1b * (-xn);
    xb = xb + n * xnb;                         // xn = x . n
    nb = nb + x * xnb;
  } else {
    xb = x2b;
  }
  if (fn > 0.0f) fnb += fcb;                   // fc = max(fn, 0)
  vctb = vtb;                                  // vt = vct - (vct . n) n
  const float pb = -dot3(n, vtb);
  nb = nb + vtb * (-p);
  vctb = vctb + n * pb;
  nb = nb + vct * pb;
  knb += fnb * delta;                          // fn = kn delta - cn vn
  deltab = kn * fnb;
  cnb -= fnb * vn;
  const float vnb = -cn * fnb;
  vrelb = n * vnb;                             // vn = vrel . n
  nb = nb + vrel * vnb;
  th.b2 += cnb * sqn + ctb * sqt;              // c = 2 beta sqrt(m* k)
  knb += cnb * S.beta2 * ms / (2.0f * sqn);
  ktb += ctb * S.beta2 * ms / (2.0f * sqt);
  th.kn += knb;
  th.kt += ktb;
  th.mu += mub;
}

struct Body { float3 x, v, w; float r, m; };

// Reverse of a pair contact (a = the particle, b = its neighbour): adds to
// a's and b's state cotangents, returns the history cotangent before the
// step.
__device__ float3 pair_vjp(const EnsSysDev& S, const Body& a, const Body& b, float3 xi, float dt,
                           float3 Fb, float3 Tb, float3 Xb, SBar& ab, SBar& bb, LawBar& th) {
  const float3 rel = a.x - b.x;
  const float dist = sqrtf(dot3(rel, rel));
  const float inv = 1.0f / dist;
  const float3 n = rel * inv;
  const float delta = overlap_pair(a.r, b.r, a.x, b.x);
  const float ms = (a.m * b.m) / (a.m + b.m);
  const float3 ua = n * (-a.r), ub = n * b.r;
  const float3 vca = a.v + cross3(a.w, ua);
  const float3 vcb = b.v + cross3(b.w, ub);
  float3 nb, vrelb, vctb, xib;
  float deltab;
  contact_vjp(S, S.mu, n, delta, ms, a.v - b.v, vca - vcb, a.r, xi, dt, Fb, Tb, Xb, nb, deltab,
              vrelb, vctb, xib, th);
  ab.v = ab.v + vctb;                          // vct = vca - vcb
  ab.w = ab.w + cross3(ua, vctb);              // vca = va + wa x ua
  nb = nb + cross3(vctb, a.w) * (-a.r);
  const float3 vcbb = vctb * (-1.0f);
  bb.v = bb.v + vcbb;                          // vcb = vb + wb x ub
  bb.w = bb.w + cross3(ub, vcbb);
  nb = nb + cross3(vcbb, b.w) * b.r;
  ab.v = ab.v + vrelb;                         // vrel = va - vb
  bb.v = bb.v - vrelb;
  float distb = -deltab;                       // delta = (ra + rb) - dist
  float3 relb = nb * inv;                      // n = rel / dist
  distb -= dot3(rel, nb) * inv * inv;
  relb = relb + rel * (distb / dist);          // dist = |rel|
  ab.x = ab.x + relb;
  bb.x = bb.x - relb;
  return xib;
}

// Reverse of a plane-wall contact of particle a (the plane is fixed).
__device__ float3 plane_vjp(const EnsSysDev& S, const EnsWallDev& W, const Body& a, float3 xi,
                            float dt, float3 Fb, float3 Tb, float3 Xb, SBar& ab, LawBar& th,
                            float& mu_wb) {
  const float3 n = W.a;
  const float delta = overlap_plane(a.r, W.a, W.r, a.x);
  const float3 ua = n * (-a.r);
  const float3 vca = a.v + cross3(a.w, ua);
  float3 nb, vrelb, vctb, xib;
  float deltab;
  LawBar tw = {0.0f, 0.0f, 0.0f, 0.0f};
  contact_vjp(S, S.mu_w, n, delta, a.m, a.v, vca, a.r, xi, dt, Fb, Tb, Xb, nb, deltab, vrelb,
              vctb, xib, tw);
  th.kn += tw.kn;
  th.kt += tw.kt;
  th.b2 += tw.b2;
  mu_wb += tw.mu;
  ab.v = ab.v + vrelb + vctb;
  ab.w = ab.w + cross3(ua, vctb);
  ab.x = ab.x + n * (-deltab);
  return xib;
}

__device__ __forceinline__ Body body(const TapeView& tv, const EnsSysDev& S, uint32_t i) {
  const float4 p = tv.pos[i], v = tv.vel[i], w = tv.angv[i];
  Body B;
  B.x = xyz4(p);
  B.v = xyz4(v);
  B.w = xyz4(w);
  B.r = p.w;
  B.m = S.dens43pi * ((p.w * p.w) * p.w);
  return B;
}

// ------------------------------------------------------------- recording
// A segment of `len` steps from step slot0: dense blocks from arena word
// `origin`, pool space after them up to `lim`.
__global__ void k_adj_seg_start(EnsTape tp, int slot0, int len, unsigned long long origin,
                                unsigned long long stride, unsigned long long lim) {
  for (int q = threadIdx.x; q < len; q += blockDim.x)
    tp.steps[slot0 + q].block = origin + (unsigned long long)q * stride;
  if (threadIdx.x == 0) {
    TapeCtl* c = tp.ctl;
    c->cur = origin + (unsigned long long)len * stride;
    c->lim = lim;
    c->lsnap = c->cur;
    c->slot = slot0 - 1;
    c->lslot = slot0;
    c->overflow = 0;
  }
}

// The current list as the list of the step about to begin (ctl->slot + 1):
// count, entries (neighbour, twin | src << 8) and, at a re-sort, the
// permutation.  twin: the neighbour's slot that holds this particle (0xff
// when the neighbour's list overflowed).
__global__ void __launch_bounds__(kThreads)
k_adj_list(EnsBufs b, EnsTape tp, int n, const StepCtl* ctl, const int* gate, int resorted,
           const int32_t* __restrict__ perm) {
  if (gate && *gate == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  TapeCtl* tc = tp.ctl;
  const int t = tc->slot + 1;
  const unsigned long long base = tc->lsnap;
  const unsigned long long lblock = tp.steps[t].lblock;
  const EnsList L = b.L[ctl->epoch & 1];
  const size_t stride = (size_t)b.stride;
  const uint32_t cnt = i < n ? L.cnt[i] : 0u;
  bool ok;
  const uint32_t off = tape_reserve(2u * cnt, &tc->cur, tc->lim, base, &tc->overflow, ok);
  if (i == 0) {
    tp.steps[t].lbase = base;
    tc->lslot = t;
  }
  if (i >= n) return;
  if (lblock != ~0ull) {
    const TapeList tl = tape_list(tp, lblock, n);
    tl.cnt[i] = cnt;
    tl.loff[i] = off;
    if (resorted) tl.perm[i] = perm[i];
  }
  if (!ok) return;
  uint2* ent = reinterpret_cast<uint2*>(tp.arena + base + off);
  for (uint32_t k = 0; k < cnt; ++k) {
    const size_t sk = (size_t)k * stride + i;
    const uint32_t j = L.idx[sk];
    const uint32_t cj = L.cnt[j];
    uint32_t tw = 0xffu;
    for (uint32_t q = 0; q < cj; ++q)
      if (L.idx[(size_t)q * stride + j] == (uint32_t)i) { tw = q; break; }
    const uint32_t src = resorted ? (uint32_t)L.src[sk] : 0xffu;
    ent[k] = make_uint2(j, tw | (src << 8));
  }
}

// Before k_adj_list: the list step's dense arrays (cnt, loff, perm) from the
// pool, ~0 when they do not fit (the overflow flag then fails the backward).
__global__ void k_adj_list_block(EnsTape tp, int n, const int* gate) {
  if (gate && *gate == 0) return;
  TapeCtl* c = tp.ctl;
  const int t = c->slot + 1;
  const unsigned long long w = tape_list_words(n);
  if (c->cur + w <= c->lim) {
    tp.steps[t].lblock = c->cur;
    c->cur += w;
  } else {
    tp.steps[t].lblock = ~0ull;
    c->overflow = 1;
  }
}

__global__ void k_adj_tick(EnsTape tp, const int* rebuilt) {
  TapeCtl* c = tp.ctl;
  const int t = c->slot + 1;
  c->slot = t;
  TapeStep& s = tp.steps[t];
  s.rb = *rebuilt != 0;
  s.lat = c->lslot;
  s.hbase = c->cur;
  c->lsnap = c->cur;
}

// --------------------------------------------------------------- reverse
// The step backwards, per particle: symplectic Euler (v' = v + (f/m + g) dt,
// x' = x + v' dt, w' = w + t/I dt) gives the cotangents of the particle's
// force and torque; then the reverse of each of its own contacts, once: its
// state, history and law-constant cotangents are kept, the share that goes
// to the neighbour is left in the slot (px, pv, pw) for k_adj_gather.
#ifndef BLAZE_ADJ_MIN_BLOCKS
#define BLAZE_ADJ_MIN_BLOCKS 5
#endif
__global__ void __launch_bounds__(kThreads, BLAZE_ADJ_MIN_BLOCKS)
k_adj_pair(EnsGeom g, EnsTape tp, int t, int n, AdjBufs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TapeStep ts = tp.steps[t];
  const TapeStep tl = tp.steps[ts.lat];
  const TapeView tv = tape_view(tp, ts.block, n);
  const TapeList lv = tape_list(tp, tl.lblock, n);
  const uint2* ent = reinterpret_cast<const uint2*>(tp.arena + tl.lbase + lv.loff[i]);
  const float* hp = reinterpret_cast<const float*>(tp.arena + ts.hbase + tv.hoff[i]);
  const uint32_t bits = __float_as_uint(tv.vel[i].w);
  const EnsSysDev& S = g.sys[bits & kSysMask];
  const Body A = body(tv, S, (uint32_t)i);
  const float inertia = (0.4f * A.m) * (A.r * A.r);
  SBar ab;
  ab.x = xyz4(a.gx[i]);
  ab.v = xyz4(a.gv[i]) + ab.x * g.dt;
  ab.w = xyz4(a.gw[i]);
  const float3 Fb = ab.v * (g.dt / A.m), Tb = ab.w * (g.dt / inertia);
  LawBar th = {0.0f, 0.0f, 0.0f, 0.0f};
  float mu_wb = 0.0f;
  const uint32_t cnt = lv.cnt[i], mask = tv.mask[i];
  // the slots in contact first (batched loads, as in the forward), then the
  // contacts and the slots that held a history, in slot order
  const uint32_t cm = tv.cmask[i];   // the contacts the forward step applied its law to
  for (uint32_t todo = cm | (mask & ((cnt >= 32u ? 0u : (1u << cnt)) - 1u)); todo;
       todo &= todo - 1u) {
    const uint32_t k = (uint32_t)(__ffs(todo) - 1);
    const size_t sl = (size_t)k * n + i;          // cotangent slot (one step)
    const bool had = (mask >> k) & 1u;
    float4 hout = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if ((cm >> k) & 1u) {
      const uint32_t j = ent[k].x;
      const float4 pb = tv.pos[j];
      const float4 vb = tv.vel[j], wb = tv.angv[j];
      Body B;
      B.x = xyz4(pb);
      B.v = xyz4(vb);
      B.w = xyz4(wb);
      B.r = pb.w;
      B.m = S.dens43pi * ((pb.w * pb.w) * pb.w);
      float3 xi = f3(0.0f, 0.0f, 0.0f);
      if (had) {
        const float* h = hp + 3 * __popc(mask & ((1u << k) - 1u));
        xi = f3(h[0], h[1], h[2]);
      }
      SBar bb;
      bb.x = f3(0.0f, 0.0f, 0.0f);
      bb.v = bb.x;
      bb.w = bb.x;
      const float3 xib = pair_vjp(S, A, B, xi, g.dt, Fb, Tb, xyz4(a.gH[sl]), ab, bb, th);
      if (had) hout = w4(xib);
      a.px[sl] = w4(bb.x);
      a.pv[sl] = w4(bb.v);
      a.pw[sl] = w4(bb.w);
    }
    if (had) a.iH[sl] = hout;
  }
  // plane walls, in the forward's order; slot nw of the output history is
  // the nw-th contact, slot q of the input the one with the same wall id
  const uint32_t wmask = bits >> kSysBits;
  float4 oh[kWallSlots];
#pragma unroll
  for (int q = 0; q < kWallSlots; ++q) oh[q] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
  if (wmask) {
    const float* hw = hp + 3 * __popc(mask);
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      if ((wmask >> q) & 1u) {
        const float* h = hw + 4 * __popc(wmask & ((1u << q) - 1u));
        oh[q] = make_float4(h[0], h[1], h[2], h[3]);
      }
  }
  float4 win[kWallSlots];
#pragma unroll
  for (int q = 0; q < kWallSlots; ++q) win[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  int nw = 0;
  for (int w = S.wall0; w < S.wall0 + S.nwall; ++w) {
    const EnsWallDev& W = g.walls[w];
    if (!(overlap_plane(A.r, W.a, W.r, A.x) > 0.0f)) continue;   // as wall_touch decides
    float3 xi = f3(0.0f, 0.0f, 0.0f);
    int qo = -1;
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      if (__float_as_int(oh[q].w) == w) { xi = xyz4(oh[q]); qo = q; }
    const float3 Xb = nw < kWallSlots ? xyz4(a.gW[(size_t)nw * n + i]) : f3(0.0f, 0.0f, 0.0f);
    const float3 xib = plane_vjp(S, W, A, xi, g.dt, Fb, Tb, Xb, ab, th, mu_wb);
#pragma unroll
    for (int q = 0; q < kWallSlots; ++q)
      if (q == qo) win[q] = w4(xib);
    ++nw;
  }
#pragma unroll
  for (int q = 0; q < kWallSlots; ++q)
    if ((wmask >> q) & 1u) a.iW[(size_t)q * n + i] = win[q];
  a.ix[i] = w4(ab.x);
  a.iv[i] = w4(ab.v);
  a.iw[i] = w4(ab.w);
  float* tr = a.th + (size_t)5 * i;
  tr[0] += th.kn;
  tr[1] += th.kt;
  tr[2] += th.b2;
  tr[3] += th.mu;
  tr[4] += mu_wb;
}

// Particle i collects, for each neighbour j in contact, the share of j's
// contact with i that k_adj_pair left in j's slot for i.
__global__ void __launch_bounds__(kThreads)
k_adj_gather(EnsTape tp, int t, int n, AdjBufs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TapeStep ts = tp.steps[t];
  const TapeStep tl = tp.steps[ts.lat];
  const TapeView tv = tape_view(tp, ts.block, n);
  const TapeList lv = tape_list(tp, tl.lblock, n);
  const uint2* ent = reinterpret_cast<const uint2*>(tp.arena + tl.lbase + lv.loff[i]);
  float3 gx = f3(0.0f, 0.0f, 0.0f), gv = gx, gw = gx;
  for (uint32_t cm = tv.cmask[i]; cm; cm &= cm - 1u) {
    const uint32_t k = (uint32_t)(__ffs(cm) - 1);
    const uint2 e = ent[k];
    const uint32_t j = e.x;
    const uint32_t q = e.y & 0xffu;
    if (q == 0xffu) continue;
    const size_t sj = (size_t)q * n + j;
    gx = gx + xyz4(a.px[sj]);
    gv = gv + xyz4(a.pv[sj]);
    gw = gw + xyz4(a.pw[sj]);
  }
  a.ix[i] = w4(xyz4(a.ix[i]) + gx);
  a.iv[i] = w4(xyz4(a.iv[i]) + gv);
  a.iw[i] = w4(xyz4(a.iw[i]) + gw);
}

// A re-sort backwards: cotangents go to the old positions and, for carried
// histories, to the old slots.
__global__ void __launch_bounds__(kThreads)
k_adj_unsort(EnsTape tp, int t, int n, AdjBufs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const TapeStep ts = tp.steps[t];
  const TapeView tv = tape_view(tp, ts.block, n);
  const TapeList tl = tape_list(tp, ts.lblock, n);
  const int io = tl.perm[i];
  a.gx[io] = a.ix[i];
  a.gv[io] = a.iv[i];
  a.gw[io] = a.iw[i];
  const uint32_t wmask = __float_as_uint(tv.vel[i].w) >> kSysBits;
#pragma unroll
  for (int q = 0; q < kWallSlots; ++q)
    if ((wmask >> q) & 1u) a.gW[(size_t)q * n + io] = a.iW[(size_t)q * n + i];
  const uint32_t cnt = tl.cnt[i];
  const uint2* ent = reinterpret_cast<const uint2*>(tp.arena + ts.lbase + tl.loff[i]);
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t s = (ent[k].y >> 8) & 0xffu;
    if (s != 0xffu) a.gH[(size_t)s * n + io] = a.iH[(size_t)k * n + i];
  }
}

// Host-layout cotangents (3 floats per particle) to and from the float4
// buffers of the sweep.
__global__ void __launch_bounds__(kThreads)
k_adj_f3_to_f4(const float* __restrict__ src, float4* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[i] = src ? make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0f)
               : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void __launch_bounds__(kThreads)
k_adj_f4_to_f3(const float4* __restrict__ src, float* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 v = src[i];
  dst[3 * i] = v.x;
  dst[3 * i + 1] = v.y;
  dst[3 * i + 2] = v.z;
}

// Law-constant cotangents summed per system in FP64: one block per system,
// each thread a strided partial sum, then a fixed tree over the block (the
// order depends only on the system's size, so repeated calls agree).
constexpr int kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads)
k_adj_sum_constants(const float* __restrict__ th, const int* __restrict__ off,
                    double* __restrict__ out) {
  __shared__ double part[5][kSumThreads];
  const int s = blockIdx.x;
  const int lo = off[s], hi = off[s + 1];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = lo + threadIdx.x; i < hi; i += kSumThreads)
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] += (double)th[5 * (size_t)i + c];
#pragma unroll
  for (int c = 0; c < 5; ++c) part[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 5; ++c) part[c][threadIdx.x] += part[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 5) out[5 * s + threadIdx.x] = part[threadIdx.x][0];
}

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

void adj_launch_seg_start(const EnsTape& tp, int slot0, int len, unsigned long long origin,
                          unsigned long long stride, unsigned long long lim, cudaStream_t st) {
  k_adj_seg_start<<<1, 256, 0, st>>>(tp, slot0, len, origin, stride, lim);
}

void adj_launch_list(const EnsBufs& b, const EnsTape& tp, int n, const StepCtl* ctl,
                     const int* gate, int resorted, const int32_t* perm, cudaStream_t st) {
  k_adj_list_block<<<1, 1, 0, st>>>(tp, n, gate);
  k_adj_list<<<nblk(n), kThreads, 0, st>>>(b, tp, n, ctl, gate, resorted, perm);
}

void adj_launch_tick(const EnsTape& tp, const int* rebuilt, cudaStream_t st) {
  k_adj_tick<<<1, 1, 0, st>>>(tp, rebuilt);
}

void adj_launch_step(const EnsGeom& g, const EnsTape& tp, int t, int n, const AdjBufs& a,
                     cudaStream_t st) {
  k_adj_pair<<<nblk(n), kThreads, 0, st>>>(g, tp, t, n, a);
  k_adj_gather<<<nblk(n), kThreads, 0, st>>>(tp, t, n, a);
}

void adj_launch_unsort(const EnsTape& tp, int t, int n, const AdjBufs& a, cudaStream_t st) {
  k_adj_unsort<<<nblk(n), kThreads, 0, st>>>(tp, t, n, a);
}

void adj_launch_f3_to_f4(const float* src, float4* dst, int n, cudaStream_t st) {
  k_adj_f3_to_f4<<<nblk(n), kThreads, 0, st>>>(src, dst, n);
}

void adj_launch_f4_to_f3(const float4* src, float* dst, int n, cudaStream_t st) {
  k_adj_f4_to_f3<<<nblk(n), kThreads, 0, st>>>(src, dst, n);
}

void adj_launch_sum_constants(const float* th, const int* off, int nsys, double* out,
                              cudaStream_t st) {
  if (nsys > 0) k_adj_sum_constants<<<nsys, kSumThreads, 0, st>>>(th, off, out);
}

}  // namespace blaze
