// poly_kernels.cu -- convex polyhedra: world-frame geometry and the fused
// polyhedron step.
//
// Compiled with -fmad=false like the sphere kernels.  Every FP32 expression
// keeps the operation order of the reference source it cites
// (Collision_Detection_Polyhedra.cuh, Utilities.cuh,
// DEM_Kernels_Compute.cuh:254-610 and 736-992, Integration.cuh:6-184), so
// contacts, forces and states equal the reference's bit for bit; the one
// exception is the half-angle sine and cosine of the quaternion update,
// evaluated here in FP64 and rounded to FP32 (see quat_step).
//
// Cases the reference leaves undefined get a defined result here and raise
// kStatusPolyUndefined:
//   * the first vertex found inside the other polyhedron has no face whose
//     plane has the vertex owner's centre on its outer side (the reference
//     then reads face -1): no vertex-face contact is reported;
//   * more than 8 vertices inside the other polyhedron (the reference's
//     8-entry arrays overflow): every vertex is counted;
//   * three or more vertices inside and none of the three candidate faces
//     confirmed by the ray test (the reference returns an uninitialised depth
//     and normal): the first candidate face is used;
//   * against a volume object: three or more vertices inside with no face
//     common to all of them (uninitialised depth and normal): the first
//     vertex's nearest face; edge pairs found but none within 0.1 of each
//     other (unset normal and points): no contact.  The per-particle contact
//     type after a test that found nothing is 0 (the reference stores an
//     unset value).
#include "poly_kernels.cuh"
#include "dem_laws.cuh"

namespace blaze {
namespace {

constexpr int kThreads = 128;

// collision classes of CollData (GPU_Memory_Transfer.cuh:41-53) that change
// what the step does with a contact
enum ContactClass : int { kNoContact = 0, kVertexFace = 1, kEdgeFace = 2, kFaceFace = 3 };

struct Hit {
  bool hit;
  int cls;
  float dis;
  float3 cp, n;
};

__device__ __forceinline__ Hit no_hit() {
  Hit h;
  h.hit = false;
  h.cls = kNoContact;
  h.dis = 0.0f;
  h.cp = f3(0.0f, 0.0f, 0.0f);
  h.n = f3(0.0f, 0.0f, 0.0f);
  return h;
}

// ---------------------------------------------------------------- quaternions
// Quaterion is (w, x, y, z) in memory (Types.h:15-21); a float4 holds it as
// (.x, .y, .z, .w) = (w, x, y, z).
struct Quat { float w, x, y, z; };

__device__ __forceinline__ Quat to_quat(float4 q) { return Quat{q.x, q.y, q.z, q.w}; }
__device__ __forceinline__ float4 to_f4(Quat q) { return make_float4(q.w, q.x, q.y, q.z); }

// Hamilton product, each component summed in the order of the reference's
// operator* (Opertators.cuh:866-875).
__device__ __forceinline__ Quat qmul(Quat a, Quat b) {
  Quat r;
  float t;
  t = a.x * b.w; t = t + a.y * b.z; t = t - a.z * b.y; r.x = t + a.w * b.x;
  t = -(a.x * b.z); t = t + a.y * b.w; t = t + a.z * b.x; r.y = t + a.w * b.y;
  t = a.x * b.y; t = t - a.y * b.x; t = t + a.z * b.w; r.z = t + a.w * b.z;
  t = -(a.x * b.x); t = t - a.y * b.y; t = t - a.z * b.z; r.w = t + a.w * b.w;
  return r;
}

// q (0, v) q*, as RotatePolyhedra forms it (Utilities.cuh:420-479)
__device__ __forceinline__ float3 rotate(Quat q, float3 v) {
  const Quat qc{q.w, -q.x, -q.y, -q.z};
  const Quat r = qmul(qmul(q, Quat{0.0f, v.x, v.y, v.z}), qc);
  return f3(r.x, r.y, r.z);
}

// ------------------------------------------------------------------ geometry
__device__ __forceinline__ float3 ld3(const float4* p) {
  const float4 a = __ldg(p);
  return f3(a.x, a.y, a.z);
}

// One particle's world-frame geometry.
struct PolyRef {
  const float4* v;      // vertices
  const float4* fn;     // face normals
  const float4* fc;     // face centroids
  const PolyShape* s;   // body-frame object (face vertex order, areas, edges)
  float3 pos;
};

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float3 shfl3(float3 v, int src) {
  return f3(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src),
            __shfl_sync(kFull, v.z, src));
}

// The face of `a` whose normal points most nearly at `p` (first of equals).
__device__ int face_towards(const PolyRef& a, float3 p) {
  const float3 d = p - a.pos;
  int best = 0;
  float bd = dot3(ld3(a.fn), d);
  for (int f = 1; f < a.s->nf; ++f) {
    const float t = dot3(ld3(a.fn + f), d);
    if (t > bd) { bd = t; best = f; }
  }
  return best;
}

// One face of is_SP_Poly_Poly: the centre of `b` on the face's outer side
// and every vertex of `b` strictly outside its plane.  The vertices are
// loaded four at a time (the test is an AND over them).
__device__ bool face_separates(const PolyRef& a, int f, const PolyRef& b) {
  const float3 n = ld3(a.fn + f), c = ld3(a.fc + f);
  if (!(dot3(n, b.pos - c) > 0.0f)) return false;
  const int nv = b.s->nv;
  int k = 0;
  for (; k + 4 <= nv; k += 4) {
    const float3 v0 = ld3(b.v + k), v1 = ld3(b.v + k + 1);
    const float3 v2 = ld3(b.v + k + 2), v3 = ld3(b.v + k + 3);
    const bool out = dot3(n, v0 - c) > 0.00000f && dot3(n, v1 - c) > 0.00000f &&
                     dot3(n, v2 - c) > 0.00000f && dot3(n, v3 - c) > 0.00000f;
    if (!out) return false;
  }
  for (; k < nv; ++k)
    if (dot3(n, ld3(b.v + k) - c) <= 0.00000f) return false;
  return true;
}

// is_SP_Poly_Poly (Utilities.cuh:105-156): does any face plane of `a`
// separate `b`?  Returns the face, or -1.  `first` (or -1) is tried before
// the others: the answer is an OR over the faces, so the order is free.
__device__ int separating_face(const PolyRef& a, const PolyRef& b, int first) {
  const int nf = a.s->nf;
  if (first >= 0 && first < nf && face_separates(a, first, b)) return first;
  for (int f = 0; f < nf; ++f)
    if (f != first && face_separates(a, f, b)) return f;
  return -1;
}

// Collision_Detection_Vertex_InPoly_3Faces (CDP:287-382): is `v` behind
// every face plane of `b`, and which three faces (with the owner's centre on
// their outer side) are nearest to it, in the reference's face order.
struct Inside {
  bool in;
  int face[3];
  float dist[3];
};

__device__ Inside vertex_inside(float3 owner, float3 v, const PolyRef& b, int reject) {
  Inside r;
  r.in = false;
  r.face[0] = r.face[1] = r.face[2] = -1;
  r.dist[0] = r.dist[1] = r.dist[2] = 10.0f;
  // a vertex outside any one face plane is not inside (the reference stops
  // at the first such face, whichever it is, and reports only that); the
  // face `reject` is the likeliest one and is tried first
  if (!(dot3(ld3(b.fn + reject), v - ld3(b.fc + reject)) < -0.0000100f)) return r;
  const int nf = b.s->nf;
  for (int f = 0; f < nf; ++f) {
    const float3 n = ld3(b.fn + f), c = ld3(b.fc + f);
    const float vd = dot3(n, v - c);
    if (!(vd < -0.0000100f)) return r;
    if (dot3(n, owner - c) > 0.0f) {
      const float ad = fabsf(vd);
      if (ad < r.dist[0]) {
        if (r.face[0] > -1) {
          if (r.face[1] > -1) { r.dist[2] = r.dist[1]; r.face[2] = r.face[1]; }
          r.dist[1] = r.dist[0]; r.face[1] = r.face[0];
        }
        r.dist[0] = ad; r.face[0] = f;
      } else if (ad < r.dist[1]) {
        if (r.face[1] > -1) { r.dist[2] = r.dist[1]; r.face[2] = r.face[1]; }
        r.dist[1] = ad; r.face[1] = f;
      } else if (ad < r.dist[2]) {
        r.dist[2] = ad; r.face[2] = f;
      }
    }
  }
  r.in = true;
  return r;
}

// is_PointOnSurface (Utilities.cuh:20-53) on face k of `b`: the fan area
// around `pt` against the face area, within tol percent.
__device__ bool on_face(const PolyRef& b, int k, float3 pt, float tol) {
  const int nv = b.s->fnv[k];
  const uint8_t* o = b.s->ford[k];
  float area = 0.000000f;
  for (int i = 0; i < nv - 1; ++i) {
    const float3 v1 = pt - ld3(b.v + o[i]);
    const float3 v2 = pt - ld3(b.v + o[i + 1]);
    area = area + 0.500000f * len3(cross3(v1, v2));
  }
  const float3 v1 = pt - ld3(b.v + o[nv - 1]);
  const float3 v2 = pt - ld3(b.v + o[0]);
  area = area + 0.500000f * len3(cross3(v1, v2));
  const float sa = b.s->farea[k];
  return (fabsf(area - sa) / sa) * 100.0000f <= tol;
}

// The ray from `from` through `to`, cut with the plane of face k of `b`:
// does the cut point lie on the face (CDP:1233-1258, repeated for every
// candidate face)?
__device__ bool ray_meets_face(const PolyRef& b, int k, float3 from, float3 to, float tol) {
  float3 ray = to - from;
  const float len = len3(ray);
  ray = f3(ray.x / len, ray.y / len, ray.z / len);
  const float3 n = ld3(b.fn + k), c = ld3(b.fc + k);
  const float dir = dot3(ray, n);
  if (!(fabsf(dir) > 0.0f)) return false;
  const float d = dot3(c - from, n) / dir;
  return on_face(b, k, from + d * ray, tol);
}

// What the vertex loop of the vertex-face test hands to its branch logic:
// how many vertices of `a` lie inside `b`, the first two (index order), the
// first one's nearest faces, the second one's second-nearest face, and the
// in-order sum of all of them.
struct VertexScan {
  int count, i0, i1, s1_face1;
  Inside s0;
  float3 sum;
};

// The vertex loop of the vertex-face test, in vertex order.
__device__ VertexScan scan_vertices(const PolyRef& a, const PolyRef& b) {
  VertexScan r;
  r.count = 0;
  r.i0 = r.i1 = r.s1_face1 = -1;
  r.s0.in = false;
  r.s0.face[0] = r.s0.face[1] = r.s0.face[2] = -1;
  r.s0.dist[0] = r.s0.dist[1] = r.s0.dist[2] = 10.0f;
  r.sum = f3(0.0f, 0.0f, 0.0f);
  const int reject = face_towards(b, a.pos);  // b's face turned to a
  const int nv = a.s->nv;
  for (int k = 0; k < nv; ++k) {
    const float3 v = ld3(a.v + k);
    const Inside t = vertex_inside(a.pos, v, b, reject);
    if (!t.in) continue;
    if (r.count == 0) { r.s0 = t; r.i0 = k; }
    else if (r.count == 1) { r.s1_face1 = t.face[1]; r.i1 = k; }
    r.sum = r.sum + v;
    ++r.count;
  }
  return r;
}

// Collision_Detection_Polyhedara_Polyhedra_VertexFaces (CDP:1154-1630),
// after the vertex loop: one vertex inside gives a vertex-face contact on
// the nearest face the ray from a's centre confirms; two, edge-face at their
// midpoint; more, face-face at their mean.
__device__ Hit resolve_vertex_face(const PolyRef& a, const PolyRef& b, const VertexScan& vs,
                                   uint32_t& st) {
  Hit h = no_hit();
  const int count = vs.count;
  if (count == 0) return h;
  const Inside& s0 = vs.s0;
  if (count > 8 || s0.face[0] < 0) st |= kStatusPolyUndefined;
  if (s0.face[0] < 0) return h;
  h.hit = true;
  const float3 va0 = ld3(a.v + vs.i0);
  const int f0 = s0.face[0];
  if (count == 1) {
    h.cls = kVertexFace;
    h.dis = s0.dist[0];
    h.n = ld3(b.fn + f0);
    h.cp = va0;
    if (s0.face[1] == -1) return h;
    if (ray_meets_face(b, f0, a.pos, va0, 0.10f)) return h;
    for (int q = 1; q < 3; ++q) {
      const int fq = s0.face[q];
      if (fq > -1 && ray_meets_face(b, fq, a.pos, va0, 0.10f)) {
        h.n = ld3(b.fn + fq);
        h.dis = s0.dist[q];
        return h;
      }
    }
    return h;  // the reference warns and keeps the nearest face
  }
  if (count == 2) {
    h.cls = kEdgeFace;
    h.cp = (va0 + ld3(a.v + vs.i1)) * 0.50f;
    h.n = ld3(b.fn + f0);
    h.dis = fabsf(dot3(h.n, h.cp - ld3(b.fc + f0)));
    if (s0.face[1] == -1 && vs.s1_face1 == -1) return h;
    for (int q = 0; q < 3; ++q) {
      const int fq = s0.face[q];
      if ((q == 0 || fq > -1) && ray_meets_face(b, fq, a.pos, h.cp, 0.10f)) {
        h.n = ld3(b.fn + fq);
        h.dis = fabsf(dot3(h.n, h.cp - ld3(b.fc + fq)));
        return h;
      }
    }
    h.n = ld3(b.fn + f0);
    h.dis = fabsf(dot3(h.n, h.cp - ld3(b.fc + f0)));
    return h;  // the reference warns and keeps the nearest face
  }
  h.cls = kFaceFace;
  h.cp = vs.sum / (float)count;
  const float tol[3] = {0.10f, 0.010f, 0.10f};
  for (int q = 0; q < 3; ++q) {
    const int fq = s0.face[q];
    if ((q == 0 || fq > -1) && ray_meets_face(b, fq, a.pos, h.cp, tol[q])) {
      h.n = ld3(b.fn + fq);
      h.dis = fabsf(dot3(h.n, h.cp - ld3(b.fc + fq)));
      return h;
    }
  }
  st |= kStatusPolyUndefined;
  h.n = ld3(b.fn + f0);
  h.dis = fabsf(dot3(h.n, h.cp - ld3(b.fc + f0)));
  return h;
}

// isPointinPoly (Utilities.cuh:60-98)
__device__ bool point_in_poly(const PolyRef& b, float3 pt) {
  const int nf = b.s->nf;
  for (int f = 0; f < nf; ++f)
    if (!(dot3(ld3(b.fn + f), pt - ld3(b.fc + f)) <= 0.000100f)) return false;
  return true;
}

// One edge pair of Collision_Detection_Polyhedra_Polyhedra_Edges
// (CDP:537-707) with the reference's arithmetic: false when the pair is
// rejected (parallel edges, a closest-point parameter outside
// [-0.01, 1.01], coincident points), else the points' distance, the edges'
// cross product and the two points.
struct EdgePair {
  float dist;
  float3 c, qa, qb;
};

__device__ __forceinline__ bool eval_edge_pair(const PolyRef& a, const PolyRef& b, int i, int j,
                                               EdgePair& out) {
  const float3 ap = ld3(a.v + a.s->edge[i][0]);
  const float3 ad = ld3(a.v + a.s->edge[i][1]) - ap;
  const float3 bp = ld3(b.v + b.s->edge[j][0]);
  const float3 bd = ld3(b.v + b.s->edge[j][1]) - bp;
  const float3 c = cross3(ad, bd);
  if (!(dot3(c, c) > 0.00000f)) return false;
  const float daa = dot3(ad, ad);
  const float3 dv = ap - bp;
  const float dbb = dot3(bd, bd);
  const float dab = dot3(ad, bd);
  const float dav = dot3(ad, dv);
  const float dbv = dot3(bd, dv);
  const float inv = __frcp_rn(dab * dab - daa * dbb);  // = 1.0f / (...), correctly rounded
  const float ta = inv * (dbb * dav - dab * dbv);
  if (!(ta >= -0.010f && ta <= 1.0100f)) return false;
  const float tb = inv * (dab * dav - daa * dbv);
  if (!(tb >= -0.0100f && tb <= 1.010f)) return false;
  const float3 qa = ap + ad * ta;
  const float3 qb = bp + bd * tb;
  const float3 d = qa - qb;
  float dist = dot3(d, d);
  if (!(dist > 0.00000f)) return false;
  out.dist = sqrtf(dist);
  out.c = c;
  out.qa = qa;
  out.qb = qb;
  return true;
}

// Distance from p to the edge (ap, ap + ad) extended by 1% at both ends
// (where the reference's closest points may lie).
__device__ __forceinline__ float extended_edge_distance(float3 p, float3 ap, float3 ad) {
  const float dd = dot3(ad, ad);
  float t = dd > 0.0f ? dot3(p - ap, ad) / dd : 0.0f;
  t = fminf(fmaxf(t, -0.01f), 1.01f);
  return len3(p - (ap + ad * t));
}

// The lanes holding the three smallest values (lowest lane among equals), or
// -1 past the values there are.
__device__ __forceinline__ void three_smallest(float v, int lane, int out[3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    float mv = v;
    int ml = lane;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const float ov = __shfl_xor_sync(kFull, mv, off);
      const int ol = __shfl_xor_sync(kFull, ml, off);
      if (ov < mv || (ov == mv && ol < ml)) { mv = ov; ml = ol; }
    }
    out[r] = mv < INFINITY ? ml : -1;
    if (lane == ml) v = INFINITY;
  }
}

// Collision_Detection_Polyhedra_Polyhedra_Edges (CDP:537-707): the closest
// pair of points between an edge of `a` and an edge of `b` (parameters
// within [-0.01, 1.01]), the first minimum in the order (edges of a outer,
// edges of b inner), normal along the edges' cross product turned towards
// `relpos`.
//
// Not every pair needs evaluating.  An edge of a at distance L from b's
// centre, with every point of b's edges within R of it, is at least L - R
// from any of them; with a rounding margin that is a lower bound for all
// pairs in its row (likewise for columns).  The exact distances of the
// 3 x 3 pairs of smallest bounds give an upper bound U on the minimum; a row
// or column whose bound exceeds U holds only pairs farther than U, so the
// minimum and the first pair attaining it lie among the remaining rows and
// columns, which the lanes evaluate exactly.  Ties go to the lowest pair
// index, as in the sequential scan.  s_idx: 64 ints of shared memory for
// this warp.
__device__ Hit edge_edge(const PolyRef& a, const PolyRef& b, float3 relpos, int lane,
                         int* s_idx) {
  Hit h = no_hit();
  const int nea = a.s->ne, neb = b.s->ne;
  if (nea <= 0 || neb <= 0) return h;
  // coordinate scale of the rounding margin
  const float M = 1.0f + a.s->rmax + b.s->rmax +
                  fmaxf(fmaxf(fmaxf(fabsf(a.pos.x), fabsf(a.pos.y)), fabsf(a.pos.z)),
                        fmaxf(fmaxf(fabsf(b.pos.x), fabsf(b.pos.y)), fabsf(b.pos.z)));
  const float marg = 1e-5f + 8e-6f * M;
  float lba = INFINITY, lbb = INFINITY;
  if (lane < nea) {
    const float3 ap = ld3(a.v + a.s->edge[lane][0]);
    const float3 ad = ld3(a.v + a.s->edge[lane][1]) - ap;
    lba = extended_edge_distance(b.pos, ap, ad) - (b.s->rmax + 0.0101f * b.s->emax) - marg;
  }
  if (lane < neb) {
    const float3 bp = ld3(b.v + b.s->edge[lane][0]);
    const float3 bd = ld3(b.v + b.s->edge[lane][1]) - bp;
    lbb = extended_edge_distance(a.pos, bp, bd) - (a.s->rmax + 0.0101f * a.s->emax) - marg;
  }
  int rs[3], cs[3];
  three_smallest(lba, lane, rs);
  three_smallest(lbb, lane, cs);
  float best = 5.0f;
  int bidx = 0x7fffffff;
  float3 nrm = f3(0.0f, 0.0f, 0.0f), qa_sel = nrm, qb_sel = nrm;
  auto consider = [&](int i, int j) {
    EdgePair e;
    if (!eval_edge_pair(a, b, i, j, e)) return;
    const int t = i * neb + j;
    if (e.dist < best || (e.dist == best && t < bidx)) {
      best = e.dist;
      bidx = t;
      nrm = e.c;
      qa_sel = e.qa;
      qb_sel = e.qb;
    }
  };
  if (lane < 9) {
    const int i = rs[lane / 3], j = cs[lane % 3];
    if (i >= 0 && j >= 0) consider(i, j);
  }
  float ub = best;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) ub = fminf(ub, __shfl_xor_sync(kFull, ub, off));
  const unsigned mr = __ballot_sync(kFull, lane < nea && !(lba > ub));
  const unsigned mc = __ballot_sync(kFull, lane < neb && !(lbb > ub));
  const unsigned below = (1u << lane) - 1u;
  if ((mr >> lane) & 1u) s_idx[__popc(mr & below)] = lane;
  if ((mc >> lane) & 1u) s_idx[32 + __popc(mc & below)] = lane;
  __syncwarp();
  const int nr = __popc(mr), nc = __popc(mc);
  for (int t = lane; t < nr * nc; t += 32) {
    const int ri = t / nc;
    consider(s_idx[ri], s_idx[32 + t - ri * nc]);
  }
  __syncwarp();
  int src = lane;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const float ob = __shfl_xor_sync(kFull, best, off);
    const int oi = __shfl_xor_sync(kFull, bidx, off);
    const int os = __shfl_xor_sync(kFull, src, off);
    if (ob < best || (ob == best && oi < bidx)) {
      best = ob;
      bidx = oi;
      src = os;
    }
  }
  if (bidx == 0x7fffffff) return h;
  nrm = shfl3(nrm, src);
  qa_sel = shfl3(qa_sel, src);
  qb_sel = shfl3(qb_sel, src);
  nrm = nrm * (1.0f / len3(nrm));
  if (len3(b.pos - qb_sel) < len3(b.pos - qa_sel) && !point_in_poly(b, qa_sel)) return h;
  h.hit = true;
  h.cls = kNoContact;  // edge-edge: no class the step treats specially
  const float s = dot3(relpos, nrm);
  if (fabsf(s) > 0.0f) {
    nrm = (s / fabsf(s)) * nrm;
    h.cp = qa_sel;
  } else {
    nrm = relpos / len3(relpos);
    h.cp = b.pos;
  }
  h.n = nrm;
  h.dis = fabsf(dot3(nrm, qb_sel - qa_sel)) + 0.000010f;
  return h;
}

// ------------------------------------------------------------ volume objects
// A volume object (lifter) seen from a polyhedral particle: its faces,
// vertices and edges are world-frame already (the host moves them).

// is_SP_VolumeObject_Poly / is_SP_Poly_VolumeObject (Utilities.cuh:212-318)
__device__ bool dobject_face_separates(const DobjDev& D, const PolyRef& a) {
  const int nv = a.s->nv;
  for (int f = 0; f < D.num_faces; ++f) {
    const float3 n = D.faces[f].normal, c = D.faces[f].centroid;
    if (!(dot3(n, a.pos - c) > 0.0f)) continue;
    bool touching = false;
    for (int k = 0; k < nv; ++k)
      if (dot3(n, ld3(a.v + k) - c) <= 0.00000f) { touching = true; break; }
    if (!touching) return true;
  }
  return false;
}

__device__ bool particle_face_separates(const PolyRef& a, const DobjDev& D) {
  const int nf = a.s->nf;
  for (int f = 0; f < nf; ++f) {
    const float3 n = ld3(a.fn + f), c = ld3(a.fc + f);
    if (!(dot3(n, D.com - c) > 0.0f)) continue;
    bool touching = false;
    for (int k = 0; k < D.num_vertex; ++k)
      if (dot3(n, D.vert[k] - c) <= 0.00000f) { touching = true; break; }
    if (!touching) return true;
  }
  return false;
}

// Collision_Detection_Vertex_InDObject_3Faces (CDP:383-476): as
// vertex_inside, with the volume object's faces and thresholds.
__device__ Inside vertex_in_dobject(float3 owner, float3 v, const DobjDev& D) {
  Inside r;
  r.in = false;
  r.face[0] = r.face[1] = r.face[2] = -1;
  r.dist[0] = r.dist[1] = r.dist[2] = 10.0f;
  for (int f = 0; f < D.num_faces; ++f) {
    const float3 n = D.faces[f].normal, c = D.faces[f].centroid;
    const float vd = dot3(n, v - c);
    if (!(vd <= 0.000010f)) return r;
    if (dot3(n, owner - c) > 0.0f) {
      const float ad = fabsf(vd);
      if (ad < r.dist[0]) {
        if (r.face[0] > -1) {
          if (r.face[1] > -1) { r.dist[2] = r.dist[1]; r.face[2] = r.face[1]; }
          r.dist[1] = r.dist[0]; r.face[1] = r.face[0];
        }
        r.dist[0] = ad; r.face[0] = f;
      } else if (ad < r.dist[1]) {
        if (r.face[1] > -1) { r.dist[2] = r.dist[1]; r.face[2] = r.face[1]; }
        r.dist[1] = ad; r.face[1] = f;
      } else if (ad < r.dist[2]) {
        r.dist[2] = ad; r.face[2] = f;
      }
    }
  }
  r.in = true;
  return r;
}

__device__ bool ray_meets_dface(const DobjDev& D, int k, float3 from, float3 to, float tol) {
  float3 ray = to - from;
  const float len = len3(ray);
  ray = f3(ray.x / len, ray.y / len, ray.z / len);
  const Surface& S = D.faces[k];
  const float dir = dot3(ray, S.normal);
  if (!(fabsf(dir) > 0.0f)) return false;
  const float d = dot3(S.centroid - from, S.normal) / dir;
  const int nv = S.num_vertex < 8 ? S.num_vertex : 8;
  return point_on_indexed_polygon(nv, D.vert, S.vertex_Order, from + d * ray, S.area, tol);
}

// Collision_Detection_Polyhedara_VolumeObject_VertexFace (CDP:1638-2002):
// vertices of the particle inside the volume object.  Face-face contact
// takes the face every such vertex has among its three nearest, at the
// smallest distance any of them records.
__device__ Hit vertex_dobject(const PolyRef& a, const DobjDev& D, uint32_t& st) {
  Hit h = no_hit();
  int count = 0, i0 = -1, i1 = -1, s1_face1 = -1;
  Inside s0;
  s0.in = false;
  s0.face[0] = -1;
  float3 sum = f3(0.0f, 0.0f, 0.0f);
  int fcnt[3] = {0, 0, 0};
  float fmin[3] = {10.0f, 10.0f, 10.0f};
  const int nv = a.s->nv;
  for (int k = 0; k < nv; ++k) {
    const float3 v = ld3(a.v + k);
    const Inside t = vertex_in_dobject(a.pos, v, D);
    if (!t.in) continue;
    if (count == 0) { s0 = t; i0 = k; }
    else if (count == 1) { s1_face1 = t.face[1]; i1 = k; }
    sum = sum + v;
    ++count;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int f = t.face[j];
      if (f > -1) {
        fcnt[f]++;
        if (t.dist[j] < fmin[f]) fmin[f] = t.dist[j];
      }
    }
  }
  if (count == 0) return h;
  if (count > 8) st |= kStatusPolyUndefined;
  const int f0 = s0.face[0];
  if (count <= 2 && f0 < 0) {
    st |= kStatusPolyUndefined;
    return h;
  }
  h.hit = true;
  const float3 va0 = ld3(a.v + i0);
  if (count == 1) {
    h.cls = kVertexFace;
    h.dis = s0.dist[0];
    h.n = D.faces[f0].normal;
    h.cp = va0;
    if (s0.face[1] == -1) return h;
    if (ray_meets_dface(D, f0, a.pos, va0, 0.1f)) return h;
    for (int s = 1; s < 3; ++s) {
      const int fs = s0.face[s];
      if (fs > -1 && ray_meets_dface(D, fs, a.pos, va0, 0.10f)) {
        h.n = D.faces[fs].normal;
        h.dis = s0.dist[s];
        return h;
      }
    }
    return h;
  }
  if (count == 2) {
    h.cls = kEdgeFace;
    h.cp = (va0 + ld3(a.v + i1)) * 0.50f;
    h.n = D.faces[f0].normal;
    h.dis = fabsf(dot3(h.n, h.cp - D.faces[f0].centroid));
    if (s0.face[1] == -1 && s1_face1 == -1) return h;
    for (int s = 0; s < 3; ++s) {
      const int fs = s0.face[s];
      if ((s == 0 || fs > -1) && ray_meets_dface(D, fs, a.pos, h.cp, 0.10f)) {
        h.n = D.faces[fs].normal;
        h.dis = fabsf(dot3(h.n, h.cp - D.faces[fs].centroid));
        return h;
      }
    }
    h.n = D.faces[f0].normal;
    h.dis = fabsf(dot3(h.n, h.cp - D.faces[f0].centroid));
    return h;
  }
  h.cls = kFaceFace;
  h.cp = sum / (float)count;
  for (int f = 0; f < D.num_faces; ++f)
    if (fcnt[f] == count) {
      h.dis = fmin[f];
      h.n = D.faces[f].normal;
      return h;
    }
  // no face common to every vertex: the reference returns an uninitialised
  // depth and normal
  st |= kStatusPolyUndefined;
  if (f0 < 0) return no_hit();
  h.dis = s0.dist[0];
  h.n = D.faces[f0].normal;
  return h;
}

// Collision_Detection_DObject_Polyhedra_Edges (CDP:716-897): edge pairs
// whose closest point on the particle's edge is nearer the particle's centre
// than the one on the volume object's; contact point their mean, normal from
// the nearest pair (within 0.1), turned against `relpos`.
__device__ Hit dobject_edges(const DobjDev& D, const PolyRef& b, float3 relpos, uint32_t& st) {
  Hit h = no_hit();
  float best = 0.10f;
  bool found = false, chosen = false;
  int count = 0;
  float3 cps = f3(0.0f, 0.0f, 0.0f), nrm = cps, qa_sel = cps, qb_sel = cps;
  const int neb = b.s->ne;
  for (int i = 0; i < D.num_edges; ++i) {
    const float3 ap = D.vert[D.edge0[i]];
    const float3 ad = D.vert[D.edge1[i]] - ap;
    const float daa = dot3(ad, ad);
    for (int j = 0; j < neb; ++j) {
      const float3 bp = ld3(b.v + b.s->edge[j][0]);
      const float3 bd = ld3(b.v + b.s->edge[j][1]) - bp;
      const float3 c = cross3(ad / len3(ad), bd / len3(bd));
      if (!(dot3(c, c) > 0.00000f)) continue;
      const float3 dv = ap - bp;
      const float dbb = dot3(bd, bd);
      const float dab = dot3(ad, bd);
      const float dav = dot3(ad, dv);
      const float dbv = dot3(bd, dv);
      const float inv = 1.00000f / (dab * dab - daa * dbb);
      const float ta = inv * (dbb * dav - dab * dbv);
      if (!(ta >= -0.010f && ta <= 1.0100f)) continue;
      const float tb = inv * (dab * dav - daa * dbv);
      if (!(tb >= -0.0100f && tb <= 1.010f)) continue;
      const float3 qa = ap + ad * ta;
      const float3 qb = bp + bd * tb;
      const float3 d = qa - qb;
      float dist = dot3(d, d);
      if (!(dist > 0.00000f)) continue;
      dist = sqrtf(dist);
      if (!(len3(b.pos - qb) > len3(b.pos - qa))) continue;
      ++count;
      cps = cps + qa;
      found = true;
      if (dist <= best) {
        best = dist;
        nrm = cross3(ad, bd);
        qa_sel = qa;
        qb_sel = qb;
        chosen = true;
      }
    }
  }
  if (!found) return h;
  if (!chosen) {  // the reference reads an unset normal and points
    st |= kStatusPolyUndefined;
    return h;
  }
  nrm = nrm * (1.0f / len3(nrm));
  h.hit = true;
  h.cls = kNoContact;
  const float s = dot3(relpos, nrm);
  if (fabsf(s) > 0.0f) {
    nrm = (-1.0f * (s / fabsf(s))) * nrm;
    h.dis = fabsf(dot3(nrm, qb_sel - qa_sel));
    h.cp = cps / (float)count;
  } else {
    nrm = (-1.0f * relpos) / len3(relpos);
    h.cp = b.pos;
    h.dis = fabsf(dot3(nrm, qb_sel - qa_sel)) + 0.000010f;
  }
  h.n = nrm;
  return h;
}

// VolumeObject_InteractionParticle for polyhedra (DEM_Kernels_Compute.cuh:
// 12-246): the first volume object in contact acts (one at a time); the
// contact type (1 vertex-face, 2 edge-edge, 0 none) is kept per particle.
__device__ void poly_dobjects(const SimParams& P, const PolyRef& A, const TypeParams& T,
                              float3 va, float3 wa, int& colltype, float3& fl, float3& tl,
                              uint32_t& st, double* el = nullptr) {
  bool outer = P.dobj[0].translating || !P.is_mill || P.rotating_wobj;
  if (!outer) outer = len3(f3(A.pos.x, A.pos.y, 0.0f) - P.cent) > (P.dobj_cyl_bound_r - 2.0f * T.radius);
  if (!outer) return;
  for (int d = 0; d < P.n_dobj; ++d) {
    const DobjDev& D = P.dobj[d];
    const float3 bv = vmul(A.pos - D.com, D.axis);
    if (!(len3(bv) < (D.bound_r + T.radius))) continue;
    if (dobject_face_separates(D, A) || particle_face_separates(A, D)) continue;
    Hit h = vertex_dobject(A, D, st);
    int ct = 1;
    if (!h.hit) {
      float3 pd = D.com;
      pd.z = A.pos.z;
      const float3 rp = pd - A.pos;
      h = dobject_edges(D, A, rp / len3(rp), st);
      ct = 2;
    }
    colltype = h.hit ? ct : 0;
    if (!h.hit) continue;
    float3 vobj = f3(0.0f, 0.0f, 0.0f);
    if (D.attached) vobj = drum_velocity(P, h.cp);
    else if (D.translating) vobj = D.velocity;
    float e = 0.0f;
    const Forces F = law_volume<true>(P, h.n, h.dis, h.cp - A.pos, wa, T, va, vobj,
                                      el ? &e : nullptr);
    fl = fl + F.trans;
    if (P.rotation) tl = tl + F.torque;
    if (el) *el += (double)e;
    break;
  }
}

// ------------------------------------------------------------- world objects
// Collision_Detection_Polyhedra_Surface + _Vertcies_Surface (CDP:85-177,
// 489-529): the centre within the bounding radius on the face's outer side,
// then the vertices behind the face plane whose projection lies on the face.
__device__ Hit poly_surface(const WallOp& op, const PolyRef& a, float bound_r) {
  Hit h = no_hit();
  if (!(dot3(op.n, a.pos - op.c) > 0.000000f)) return h;
  if (!(dot3(op.n, a.pos - op.c) <= bound_r)) return h;
  int count = 0;
  float dmax = 0.0f;
  bool any = false;
  float3 cp = f3(0.0f, 0.0f, 0.0f);
  const int nv = a.s->nv;
  for (int k = 0; k < nv; ++k) {
    const float3 v = ld3(a.v + k);
    const float vd = dot3(op.n, v - op.c);
    if (!(vd < 0.000000f)) continue;
    const float3 hp = v + fabsf(vd) * op.n;
    if (!point_on_polygon(op.nv, op.v, hp, op.area, op.tol)) continue;
    ++count;
    cp = cp + hp;
    if (fabsf(vd) > dmax) {
      any = true;
      dmax = fabsf(vd);
    }
    if (count > 2) {  // face on face: no moment, contact at the centre
      h.hit = true; h.cls = kFaceFace; h.n = op.n; h.dis = dmax; h.cp = a.pos;
      return h;
    }
  }
  if (!any) return h;
  h.hit = true;
  h.cls = count == 1 ? kVertexFace : kEdgeFace;
  h.n = op.n;
  h.dis = dmax;
  h.cp = cp / (float)count;
  return h;
}

// Collision_Detection_Polyhedra_Cylinder (CDP:2010-2132): vertices beyond
// the drum radius; depth = their mean radial excess (the reference scales by
// a double reciprocal of the count), face-face capped at 0.001.
__device__ Hit poly_cylinder(const WallOp& op, const PolyRef& a, float bound_r) {
  Hit h = no_hit();
  const float3 pv = vmul(a.pos, op.axis) - op.cbot;
  if (!(len3(pv) + bound_r > op.radius)) return h;
  float dis = 0.0f;
  int count = 0;
  float3 sp = f3(0.0f, 0.0f, 0.0f);
  float3 nrm = f3(-pv.x, -pv.y, -pv.z);
  nrm = nrm * (1.0f / len3(nrm));
  const int nv = a.s->nv;
  for (int k = 0; k < nv; ++k) {
    const float3 v = ld3(a.v + k);
    const float rc = len3(vmul(v, op.axis) - op.cbot);
    if (!(rc > op.radius)) continue;
    ++count;
    sp = sp + v;
    dis = dis + (rc - op.radius);
    if (count > 2) {
      dis = (float)((double)dis * (1.0 / (double)(float)count));
      h.hit = true; h.cls = kFaceFace; h.n = nrm; h.dis = fminf(0.00100f, fabsf(dis));
      h.cp = a.pos;
      return h;
    }
  }
  if (count == 0) return h;
  h.hit = true;
  h.n = nrm;
  dis = (float)((double)dis * (1.0 / (double)(float)count));
  if (count == 2) {
    h.cls = kEdgeFace;
    h.cp = sp / (float)count;
    h.dis = fabsf(dis);
  } else {
    h.cls = kVertexFace;
    h.cp = sp;
    h.dis = dis;
  }
  return h;
}

// Collision_Detection_Vertcies_Plane (CDP:6-75), used for the drum's end
// plates: every vertex behind the plane; depth of the deepest.
__device__ Hit vertices_plane(const PolyRef& a, float3 n, float3 c) {
  Hit h = no_hit();
  int count = 0;
  float dmax = 0.0f;
  float3 cp = f3(0.0f, 0.0f, 0.0f);
  const int nv = a.s->nv;
  for (int k = 0; k < nv; ++k) {
    const float3 v = ld3(a.v + k);
    const float vd = dot3(n, v - c);
    if (!(vd < 0.000000f)) continue;
    ++count;
    cp = cp + v;
    if (fabsf(vd) > dmax) dmax = fabsf(vd);
  }
  if (count == 0) return h;
  h.hit = true;
  h.cls = count == 2 ? kEdgeFace : kFaceFace;  // the reference's if/else leaves one vertex as face-face
  h.cp = cp / (float)count;
  h.n = n;
  h.dis = dmax;
  return h;
}

// WorldObject_InteractionParticle for polyhedra (DEM_Kernels_Compute.cuh:
// 254-610).  The reference keeps one contact record across the loop and
// assigns nothing for an infinite plane (it has no polyhedron method), so a
// plane applies the record the previous world-object step left behind.
__device__ void poly_walls(const SimParams& P, const WallOp* __restrict__ ops, const PolyRef& A,
                           const TypeParams& T, float3 va, float3 wa, float3& fw, float3& tw,
                           double* es = nullptr) {
  Hit last = no_hit();
  float e = 0.0f;
  float* ep = es ? &e : nullptr;
  for (int q = 0; q < P.n_ops; ++q) {
    const WallOp& op = ops[q];
    if (op.kind == kOpFace || op.kind == kOpPlane) {
      if (op.kind == kOpFace) last = poly_surface(op, A, T.radius);
      if (!last.hit) continue;
      Forces F;
      if (P.rotating_wobj && P.cyl_rot)
        F = law_moving_surface<true>(P, last.n, last.dis, last.cp - A.pos, wa, T, va,
                                     drum_velocity(P, last.cp), ep);
      else
        F = law_static_surface(P, va, last.n, last.dis, last.cp - A.pos, wa, T, ep);
      fw = fw + F.trans;
      if (P.rotation && last.cls != kFaceFace) tw = tw + F.torque;
      if (es) *es += (double)e;
    } else if (op.kind == kOpCylinder) {
      last = poly_cylinder(op, A, T.radius);
      if (!last.hit) continue;
      Forces F;
      if (P.cyl_rot)
        F = law_moving_surface<true>(P, last.n, last.dis, last.cp - A.pos, wa, T, va,
                                     drum_velocity(P, last.cp), ep);
      else
        F = law_static_surface(P, va, last.n, last.dis, last.cp - A.pos, wa, T, ep);
      fw = F.trans;
      if (P.rotation && last.cls != kFaceFace) tw = tw + F.torque;
      if (es) *es += (double)e;
    } else {  // end plates (Collision_Response_EndPlate_Particle: no torque)
      last = vertices_plane(A, op.n, op.c);
      if (!last.hit) continue;
      fw = law_end_plate(va, last.n, last.dis, T);
      if (P.rotation) tw = tw + f3(0.0f, 0.0f, 0.0f);
    }
  }
}

// -------------------------------------------------------------- integration
// Get_Angular_Acc (Utilities.cuh:486-608): I(t)^-1 tau with
// I(t)^-1 = R(q) I0^-1 R(q)^T, sums in the reference's loop order.
__device__ float3 angular_acc(Quat q, const float* __restrict__ I0, float3 tau) {
  float R[9];
  R[0] = q.w * q.w + q.x * q.x - q.y * q.y - q.z * q.z;
  R[1] = 2.0f * q.x * q.y - 2.0f * q.w * q.z;
  R[2] = 2.0f * q.x * q.z + 2.0f * q.w * q.y;
  R[3] = 2.0f * q.x * q.y + 2.0f * q.w * q.z;
  R[4] = q.w * q.w - q.x * q.x + q.y * q.y - q.z * q.z;
  R[5] = 2.0f * q.y * q.z - 2.0f * q.w * q.x;
  R[6] = 2.0f * q.x * q.z - 2.0f * q.w * q.y;
  R[7] = 2.0f * q.y * q.z + 2.0f * q.w * q.x;
  R[8] = q.w * q.w - q.x * q.x - q.y * q.y + q.z * q.z;
  float I[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) I[k] = __ldg(I0 + k);
  float RI[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float s = 0.0f;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += R[r * 3 + k] * I[k * 3 + c];
      RI[r * 3 + c] = s;
    }
  float W[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float s = 0.0f;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += RI[k * 3 + c] * R[k * 3 + r];
      W[r * 3 + c] = s;
    }
  const float t[3] = {tau.x, tau.y, tau.z};
  float a[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) s += W[r * 3 + k] * t[k];
    a[r] = s;
  }
  return f3(a[0], a[1], a[2]);
}

// Orientation update of Integrate_Euler_NonSymmetry (Integration.cuh:
// 132-164): dq = (cos(|w| dt / 2), sin(|w| dt / 2) w / |w|),
// q <- normalise(dq q), or dq when that lands on w <= -1.  The reference
// calls the FP32 cosine and sine; here both are the FP64 library functions
// rounded to FP32 (the correctly rounded FP32 values except within ~1e-16
// relative of a rounding boundary).  The sine's products with w / |w| are
// exact in the reference's FP64 and rounded once, the same as FP32 products.
__device__ float4 quat_step(float4 q4, float3 w, float dt) {
  float mag = dot3(w, w);
  Quat dq{1.000000f, 0.000000f, 0.000000f, 0.000000f};
  if (mag > 0.000000f) {
    mag = sqrtf(mag);
    const float3 dir = w / mag;
    const float half = 0.5000f * mag * dt;
    dq.w = (float)cos((double)half);
    const float s = (float)sin((double)half);
    dq.x = s * dir.x;
    dq.y = s * dir.y;
    dq.z = s * dir.z;
  }
  const Quat p = qmul(dq, to_quat(q4));
  const float sq = p.w * p.w + p.x * p.x + p.y * p.y + p.z * p.z;
  const float inv = sq > 0.0f ? 1.0f / sqrtf(sq) : 0.0f;
  const Quat qn{p.w * inv, p.x * inv, p.y * inv, p.z * inv};
  return to_f4(qn.w <= -1.00000f ? dq : qn);
}

// ------------------------------------------------------------------- kernels
__global__ void __launch_bounds__(kThreads)
k_poly_geom(const PolyShape* __restrict__ shapes, PolyGeom g, StateBuf in_plain,
            StateBuf in_sorted, OrderBuf ob, int rotation, const StepCtl* ctl,
            const int* rebuilt) {
  const int ke = g.kv > g.kf ? g.kv : g.kf;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / ke);
  const int e = (int)(t - (long long)i * ke);
  if (i >= ctl->n_cur) return;
  const StateBuf in = *rebuilt ? in_sorted : in_plain;
  const float3 p = xyz(in.pos[i]);
  const int ty = __float_as_int(in.vel[i].w) & (kMaxTypes - 1);
  const PolyShape& S = shapes[ty];
  Quat q{1.0f, 0.0f, 0.0f, 0.0f};
  if (rotation) q = to_quat(((ctl->epoch & 1) ? ob.ornt[1] : ob.ornt[0])[i]);
  if (e < S.nv) {
    const float3 lv = xyz(S.vert[e]);
    const float3 v = (rotation ? rotate(q, lv) : lv) + p;
    g.vert[(size_t)i * g.kv + e] = make_float4(v.x, v.y, v.z, 0.0f);
  }
  if (e < S.nf) {
    const float3 n = xyz(S.fnorm[e]);
    const float3 c = xyz(S.fcent[e]);
    const float3 nw = rotation ? rotate(q, n) : n;
    const float3 cw = (rotation ? rotate(q, c) : c) + p;
    g.fnorm[(size_t)i * g.kf + e] = make_float4(nw.x, nw.y, nw.z, 0.0f);
    g.fcent[(size_t)i * g.kf + e] = make_float4(cw.x, cw.y, cw.z, 0.0f);
  }
}

// ------------------------------------------------------------ narrow phase
// The pairs of a step go through the reference's tests in three passes,
// each with the parallelism its test wants; a pass records its verdict per
// neighbour slot (slot = k * stride + i) and queues the slots the next test
// must see.  Every pair is evaluated with the reference's arithmetic, and the
// step sums the contacts in slot order, so the results do not depend on the
// order in which queued slots are taken.
enum SlotState : uint8_t { kSlotNone = 0, kSlotVertex = 1, kSlotContact = 2, kSlotEdge = 3 };

__device__ __forceinline__ PolyRef poly_ref(const PolyGeom& g, const PolyShape* shapes, int i,
                                            float4 p4, float4 v4) {
  const int t = __float_as_int(v4.w) & (kMaxTypes - 1);
  return PolyRef{g.vert + (size_t)i * g.kv, g.fnorm + (size_t)i * g.kf,
                 g.fcent + (size_t)i * g.kf, shapes + t, xyz(p4)};
}

__device__ __forceinline__ void store_contact(const PolyPairs& pp, uint32_t slot, const Hit& h) {
  pp.con[2 * (size_t)slot] = make_float4(h.n.x, h.n.y, h.n.z, h.dis);
  pp.con[2 * (size_t)slot + 1] = make_float4(h.cp.x, h.cp.y, h.cp.z, 0.0f);
  pp.status[slot] = kSlotContact;
}

__device__ __forceinline__ void flag_status_warp(StepCtl* ctl, uint32_t bits) {
  const unsigned m = __activemask();
  const uint32_t all = __reduce_or_sync(m, bits);
  if (all && (threadIdx.x & 31) == (__ffs(m) - 1)) atomicOr(&ctl->status, all);
}

// Pass 1, one thread per filled neighbour slot (the contact-list kernel's
// flat list): bounding spheres (Collision_Detection_BroadPhase.cuh:369-384;
// a no-op in reference mode, where the list holds overlapping pairs only),
// then the separating face planes of A against B and of B against A
// (DEM_Kernels_Compute.cuh:842-860), starting from the face that separated
// the slot's pair last step.  Every thread runs the same number of rounds so
// the block can append its queue entries at once.
__global__ void __launch_bounds__(kThreads)
k_poly_sep(const PolyShape* __restrict__ shapes, PolyGeom g, StateBuf in_plain,
           StateBuf in_sorted, NbrList nl, const int* rebuilt, PolyPairs pp) {
  __shared__ int s_cnt, s_base;
  const int total = *nl.flat_n;
  const int nthreads = gridDim.x * blockDim.x;
  const int rounds = (total + nthreads - 1) / nthreads;
  const StateBuf in = *rebuilt ? in_sorted : in_plain;
  for (int r = 0; r < rounds; ++r) {
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const int e = r * nthreads + blockIdx.x * blockDim.x + threadIdx.x;
    bool queue = false;
    uint32_t slot = 0;
    if (e < total) {
      slot = nl.flat[e];
      const int i = (int)(slot % (uint32_t)nl.stride);
      const int j = (int)nl.idx[slot];
      const float4 pa4 = in.pos[i], pb4 = __ldg(in.pos + j);
      uint8_t v = kSlotNone;
      if (len3(xyz(pa4) - xyz(pb4)) - (pa4.w + pb4.w) < 0.0f) {
        const PolyRef A = poly_ref(g, shapes, i, pa4, in.vel[i]);
        const PolyRef B = poly_ref(g, shapes, j, pb4, __ldg(in.vel + j));
        // the face that separated this slot's pair last step, if any, first
        const int hint = pp.hint[slot];
        int hint_b = hint != 0xff && (hint & 0x80) ? hint & 0x3f : -1;
        int f = separating_face(A, B, hint != 0xff && !(hint & 0x80) ? hint : -1);
        int newhint = f >= 0 ? f : 0xff;
        if (f < 0) {
          f = separating_face(B, A, hint_b);
          newhint = f >= 0 ? (0x80 | f) : 0xff;
        }
        if (newhint != hint) pp.hint[slot] = (uint8_t)newhint;
        if (f < 0) {
          v = kSlotVertex;
          queue = true;
        }
      }
      pp.status[slot] = v;
    }
    int off = 0;
    if (queue) off = atomicAdd(&s_cnt, 1);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) s_base = atomicAdd(&pp.counts[0], s_cnt);
    __syncthreads();
    if (queue) pp.qv[s_base + off] = slot;
  }
}

// Pass 2, one thread per queued slot: vertices of A in B, then of B in A
// with the normal reversed (DEM_Kernels_Compute.cuh:862-890).  Slots
// without a vertex inside queue for the edge test.  Every thread runs the
// same number of rounds so the block can append its queue entries at once.
__global__ void __launch_bounds__(kThreads)
k_poly_vf(const PolyShape* __restrict__ shapes, PolyGeom g, StateBuf in_plain,
          StateBuf in_sorted, NbrList nl, StepCtl* ctl, const int* rebuilt, PolyPairs pp) {
  __shared__ int s_cnt, s_base;
  const int total = pp.counts[0];
  const int nthreads = gridDim.x * blockDim.x;
  const int rounds = (total + nthreads - 1) / nthreads;
  const StateBuf in = *rebuilt ? in_sorted : in_plain;
  uint32_t st = 0;
  for (int r = 0; r < rounds; ++r) {
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const int e = r * nthreads + blockIdx.x * blockDim.x + threadIdx.x;
    bool queue = false;
    uint32_t slot = 0;
    if (e < total) {
      slot = pp.qv[e];
      const int i = (int)(slot % (uint32_t)nl.stride);
      const int j = (int)nl.idx[slot];
      const float4 pa4 = in.pos[i], pb4 = in.pos[j];
      const PolyRef A = poly_ref(g, shapes, i, pa4, in.vel[i]);
      const PolyRef B = poly_ref(g, shapes, j, pb4, in.vel[j]);
      Hit h = resolve_vertex_face(A, B, scan_vertices(A, B), st);
      if (!h.hit) {
        h = resolve_vertex_face(B, A, scan_vertices(B, A), st);
        h.n = h.n * -1.0f;
      }
      if (h.hit) {
        store_contact(pp, slot, h);
      } else {
        pp.status[slot] = kSlotEdge;
        queue = true;
      }
    }
    int off = 0;
    if (queue) off = atomicAdd(&s_cnt, 1);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) s_base = atomicAdd(&pp.counts[1], s_cnt);
    __syncthreads();
    if (queue) pp.qe[s_base + off] = slot;
  }
  flag_status_warp(ctl, st);
}

// Pass 3, one warp per queued slot: the edge-edge test, depth capped at
// 0.025 r_A (DEM_Kernels_Compute.cuh:894-915).
__global__ void __launch_bounds__(kThreads)
k_poly_ee(const SimParams* __restrict__ Pg, const PolyShape* __restrict__ shapes, PolyGeom g,
          StateBuf in_plain, StateBuf in_sorted, NbrList nl, const int* rebuilt, PolyPairs pp) {
  __shared__ int s_idx[kThreads / 32][64];
  const int total = pp.counts[1];
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  const StateBuf in = *rebuilt ? in_sorted : in_plain;
  for (int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < total; e += nwarps) {
    const uint32_t slot = pp.qe[e];
    const int i = (int)(slot % (uint32_t)nl.stride);
    const int j = (int)nl.idx[slot];
    const float4 pa4 = in.pos[i], pb4 = in.pos[j], va4 = in.vel[i];
    const PolyRef A = poly_ref(g, shapes, i, pa4, va4);
    const PolyRef B = poly_ref(g, shapes, j, pb4, in.vel[j]);
    const float3 d = A.pos - B.pos;
    Hit h = edge_edge(A, B, d / len3(d), lane, s_idx[threadIdx.x >> 5]);
    if (h.hit) h.dis = fminf(0.025f * Pg->types[__float_as_int(va4.w) & (kMaxTypes - 1)].radius, h.dis);
    if (lane == 0) {
      if (h.hit) store_contact(pp, slot, h);
      else pp.status[slot] = kSlotNone;
    }
  }
}

// The polyhedron step: the particle-particle sum of
// Kernel_ParticleInteraction_Polyhedra_NonSymmetry (DEM_Kernels_Compute.cuh:
// 736-992) over the contacts the passes found, in slot order, with the
// reference's depth limits; VolumeObject_InteractionParticle,
// WorldObject_InteractionParticle and Integrate_Euler_NonSymmetry with the
// quaternion update.  One thread per particle.
template <bool kCapture, bool kEnergy>
__global__ void __launch_bounds__(kThreads)
k_poly_step(const SimParams* __restrict__ Pg, const PolyShape* __restrict__ shapes, PolyGeom g,
            const WallOp* __restrict__ ops, StateBuf in_plain, StateBuf in_sorted, StateBuf out,
            OrderBuf ob, int n_max, NbrList nl, PolyPairs pp, StepCtl* ctl, StepLink link,
            ForceCapture cap, double* eb) {
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
  uint32_t st = (ta < 0 || ta >= P.n_types) ? kStatusTypeRange : 0u;
  const int tA = ta & (kMaxTypes - 1);
  const TypeParams& TA = sT[tA];
  const float ma = TA.mass, ra = pa4.w;
  const PolyRef A{g.vert + (size_t)i * g.kv, g.fnorm + (size_t)i * g.kf,
                  g.fcent + (size_t)i * g.kf, shapes + tA, pa};

  // particle-particle
  float3 f = P.gravity * ma;
  float3 fl = f3(0.0f, 0.0f, 0.0f);
  double e_pp = 0.0, e_lift = 0.0, e_surf = 0.0;
  float ec = 0.0f;
  const int cnt = (int)nl.cnt[i];
  for (int k = 0; k < cnt; ++k) {
    const size_t slot = (size_t)k * nl.stride + i;
    if (pp.status[slot] != kSlotContact) continue;
    const int j = (int)nl.idx[slot];
    const float4 pb4 = __ldg(in.pos + j);
    const float3 pb = xyz(pb4);
    const float4 vb4 = __ldg(in.vel + j);
    const float3 vb = xyz(vb4), wb = xyz(__ldg(in.angv + j));
    const int tb = __float_as_int(vb4.w);
    const float4 c0 = pp.con[2 * slot], c1 = pp.con[2 * slot + 1];
    float3 n = xyz(c0), cp = xyz(c1);
    float dis = c0.w;
    const float3 rvel = va - vb;
    const float3 d = pa - pb;
    const float3 relpos = d / len3(d);
    // depth limits of the reference (DEM_Kernels_Compute.cuh:917-950)
    if (dis > 0.1500f * TA.radius) {
      n = relpos / len3(relpos);
      dis = 0.025f * TA.radius;
      cp = pa;
    }
    if (dis > 0.0500f * TA.radius) {
      n = relpos / len3(relpos);
      dis = len3(rvel) > 50.0f ? 0.010f * TA.radius : 0.0030f * TA.radius;
      cp = pa;
    }
    const PP_Parms& ppar = TA.pp[tb < kMaxPP ? tb : 0];
    const Forces F = law_pp<true>(P, rvel, n, dis, cp - pa, cp - pb, wa, wb, ppar, va, vb, ma,
                                  sT[tb & (kMaxTypes - 1)].mass, kEnergy ? &ec : nullptr);
    f = f + F.trans;
    fl = fl + F.torque;
    if (kEnergy) e_pp += (double)ec;
  }
  const float3 f_pp = f;
  const float3 t_pp = P.rotation ? fl : f3(0.0f, 0.0f, 0.0f);

  // volume objects
  float3 f_l = f3(0.0f, 0.0f, 0.0f), t_l = f3(0.0f, 0.0f, 0.0f);
  if (P.n_dobj > 0) {
    int* lift = (ctl->epoch & 1) ? ob.lift[1] : ob.lift[0];
    int colltype = 0;
    poly_dobjects(P, A, TA, va, wa, colltype, f_l, t_l, st, kEnergy ? &e_lift : nullptr);
    lift[i] = colltype;
  }

  // world objects
  float3 f_w = f3(0.0f, 0.0f, 0.0f), t_w = f3(0.0f, 0.0f, 0.0f);
  poly_walls(P, ops, A, TA, va, wa, f_w, t_w, kEnergy ? &e_surf : nullptr);
  if (!P.rotation) t_w = f3(0.0f, 0.0f, 0.0f);
  if (kEnergy) {
    eb[i] = e_pp;
    eb[(size_t)n_max + i] = e_lift;
    eb[2 * (size_t)n_max + i] = e_surf;
  }

  // Integrate_Euler_NonSymmetry (Integration.cuh:6-184), polyhedra
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
    float4* qarr = (ctl->epoch & 1) ? ob.ornt[1] : ob.ornt[0];
    const float4 q0 = qarr[i];
    if (dot3(tl, tl) > 0.0f) {
      const float3 aa = angular_acc(to_quat(q0), shapes[tA].inertia, tl);
      w = w + aa * P.dt;
      w = w - w * P.roll_res;
    }
    float4 q1 = quat_step(q0, w, P.dt);
    if (P.mode2d) { q1.y = 0.0f; q1.z = 0.0f; }  // x and y of (w, x, y, z)
    qarr[i] = q1;
    if (P.mode2d) { w.x = 0.0f; w.y = 0.0f; }
  }
  float path = wa4.w;
  if (P.skin > 0.0f) path = path + len3(v) * P.dt;
  out.pos[i] = make_float4(p.x, p.y, p.z, ra);
  out.vel[i] = make_float4(v.x, v.y, v.z, va4.w);
  out.angv[i] = make_float4(w.x, w.y, w.z, path);
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) st |= kStatusNonFinite;

  // Verlet-list validity on the bounding spheres, as for spheres
  {
    const unsigned m = __activemask();
    const bool need = list_needs_rebuild(P.skin, link, ctl->exact, path, len3(v), ctl, st);
    const unsigned b = __ballot_sync(m, need);
    if (b && (threadIdx.x & 31) == (__ffs(m) - 1)) {
      if (link.has_next_h) cudaGraphSetConditional(link.next_h, 1u);
      else atomicExch(&ctl->rebuild_req, 1);
    }
  }
  flag_status_warp(ctl, st);

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

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

void launch_poly_geom(const PolyShape* shapes, PolyGeom g, const StateBuf& in_plain,
                      const StateBuf& in_sorted, const OrderBuf& ob, int n_max, int rotation,
                      const StepCtl* ctl, const int* rebuilt, cudaStream_t st) {
  const long long ke = g.kv > g.kf ? g.kv : g.kf;
  k_poly_geom<<<blocks_for((long long)n_max * ke), kThreads, 0, st>>>(shapes, g, in_plain,
                                                                       in_sorted, ob, rotation,
                                                                       ctl, rebuilt);
}

int launch_poly_pairs(const SimParams* dp, const PolyShape* shapes, PolyGeom g,
                      const StateBuf& in_plain, const StateBuf& in_sorted, int n_max, NbrList nl,
                      StepCtl* ctl, const int* rebuilt, PolyPairs pp, cudaStream_t st) {
  cudaMemsetAsync(pp.counts, 0, 2 * sizeof(int), st);
  k_poly_sep<<<pp.grid_s, kThreads, 0, st>>>(shapes, g, in_plain, in_sorted, nl, rebuilt, pp);
  k_poly_vf<<<pp.grid_v, kThreads, 0, st>>>(shapes, g, in_plain, in_sorted, nl, ctl, rebuilt, pp);
  k_poly_ee<<<pp.grid_e, kThreads, 0, st>>>(dp, shapes, g, in_plain, in_sorted, nl, rebuilt, pp);
  return 3;
}

void launch_poly_step(const SimParams* dp, const PolyShape* shapes, PolyGeom g,
                      const WallOp* ops, const StateBuf& in_plain, const StateBuf& in_sorted,
                      const StateBuf& out, const OrderBuf& ob, int n_max, NbrList nl,
                      PolyPairs pp, StepCtl* ctl, StepLink link, const ForceCapture* cap,
                      double* eb, cudaStream_t st) {
  const ForceCapture c = cap ? *cap : ForceCapture{};
  const int gr = blocks_for(n_max);
#define POLY_STEP(C, E)                                                                      \
  k_poly_step<C, E><<<gr, kThreads, 0, st>>>(dp, shapes, g, ops, in_plain, in_sorted, out, ob, \
                                             n_max, nl, pp, ctl, link, c, eb)
  if (eb) {
    if (cap) POLY_STEP(true, true);
    else POLY_STEP(false, true);
  } else {
    if (cap) POLY_STEP(true, false);
    else POLY_STEP(false, false);
  }
#undef POLY_STEP
}

}  // namespace blaze
