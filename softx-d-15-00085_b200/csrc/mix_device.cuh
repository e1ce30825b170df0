// mix_device.cuh -- convex polyhedra among the spheres of an ensemble system
// (the ball mill's mixed charge of steel balls and rocks).
//
// The reference holds either spheres or polyhedra in a run, never both
// (KSimulationData.cpp:129-141), and meets polyhedra with its own vertex-face
// and edge-edge passes (DEM_Kernels_Compute.cuh:752-1031).  Here a
// polyhedron is a convex hull of at most 16 vertices and 28 triangular faces
// in its body frame (centre of mass at the origin) with its mass and inertia
// tensor, carried through the ensemble's broad phase as its bounding sphere,
// and met by:
//   sphere - polyhedron   the closest point of the hull to the sphere's centre
//                         (the face of largest signed distance, else the
//                         nearest point of the faces the centre lies outside)
//   polyhedron pairs      the separating-axis test over both hulls' face
//                         normals and the cross products of the edge pairs
//                         that form a face of the Minkowski difference
//                         (Gregorius, "The Separating Axis Test between Convex
//                         Polyhedra", GDC 2013): the axis of least penetration
//                         is the contact normal, faces preferred over edges
//   polyhedron - triangle the same test against the triangle as a flat hull
//                         (two faces, three edges, every edge pair's axis with
//                         full support extents)
//   polyhedron - plane    the deepest vertex below the plane
// All of it in FP64 from the FP32 state: a resting contact's overlap is
// ~1e-6 cm against vertex offsets of ~1 cm and positions of ~50 cm.  The
// contact point is the mean of the penetrating vertices weighted by their
// depths (a face axis: it moves continuously as vertices enter and leave,
// and shifts toward the deeper side under an off-centre load, as a pressure
// distribution would) or the midpoint of the closest points of the two
// edges (an edge axis).  The law
// is the ensemble's linear law with tangential history, evaluated with the
// contact point's relative velocity, without rolling friction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ens_device.cuh"
#include "ens_kernels.cuh"

namespace blaze {

constexpr int kMixMaxV = 16;     // vertices of a shape
constexpr int kMixMaxF = 28;     // triangular faces (2 V - 4)
constexpr int kMixMaxE = 42;     // edges (3 V - 6)
constexpr int kMixSlots = 64;    // neighbour slots of a polyhedron
constexpr int kMixWallSlots = 16; // wall contacts (tangential histories) of a polyhedron

struct MixShapeDev {
  int nv, nf, ne, pad;
  float mass;        // kg
  float rb;          // bounding radius about the centre of mass, cm
  float inertia[9];  // body frame, kg cm^2, row-major
  float iinv[9];     // its inverse
};

// One copy of the polyhedra's neighbour lists, slot-major over polyhedron
// ids (slot k of polyhedron p at k * npoly + p); a 64-bit mask of active
// tangential histories per polyhedron (mlo: slots 0-31, mhi: 32-63).  A pair
// of polyhedra that an axis separated stays apart along it for a while:
// that axis is tried first the next step (same answer as the full test when
// it still separates them, since the full test takes the largest
// separation).
struct MixList {
  uint32_t* idx;
  uint32_t* cnt;
  uint32_t* mlo;
  uint32_t* mhi;
  float* hx;
  float* hy;
  float* hz;
  int* sep;     // per slot: the axis that last separated a polyhedron pair
                // (kind << 16 | index: 0 a face of A, 1 a face of B, 2 an edge
                // pair; A the lower id), -1 none
};

// Everything about the polyhedra.  Per shape: bv (kMixMaxV body vertices),
// bn (kMixMaxF body unit normals, FP64), faces (kMixMaxF vertex triples,
// counter-clockwise seen from outside), edges (kMixMaxE: vertex i < j, faces
// f1 < f2).  Per polyhedron id: its shape, orientation (w, x, y, z), memory
// position, path since the last re-sort, and world-frame geometry rebuilt
// every step: gv (vertex offsets from the centre) and gf (unit normal,
// offset h: the face plane is n . x = h relative to the centre), FP64; its
// wall histories (wh: kMixWallSlots of (xi, wall id), wn in use), kept per
// id (a polyhedron's vel4.w carries no wall-history mask).
struct MixBufs {
  const MixShapeDev* shapes;
  const float4* bv;
  const double4* bn;
  const uchar4* faces;
  const uchar4* edges;
  const int* shape_of;
  float4* quat;
  int* pat;
  float* ppath;
  double4* gv;
  double4* gf;
  float4* wh;
  int* wn;
  float4* sf;           // per polyhedron slot: force on the sphere there (w = 1: contact)
  float4* st;           // and its torque
  uint8_t* twin;        // per sphere slot (sphere list layout): see MixView
  MixList L[2];
  int npoly;
};

// ------------------------------------------------------------ FP64 vectors
__device__ __forceinline__ double3 dv(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 dxyz(double4 a) { return dv(a.x, a.y, a.z); }
__device__ __forceinline__ double3 dadd(double3 a, double3 b) { return dv(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 dscale(double3 a, double s) { return dv(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double3 dneg(double3 a) { return dv(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double3 dcross(double3 a, double3 b) {
  return dv(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 to_f3(double3 a) { return f3((float)a.x, (float)a.y, (float)a.z); }

// The rotation of the unit quaternion q4 = (w, x, y, z), formed in FP64 from
// the FP32 components with the norm divided out (orthogonal whatever the
// FP32 rounding of |q|).
__device__ __forceinline__ void mix_rotation(float4 q4, double* R) {
  const double w = q4.x, x = q4.y, y = q4.z, z = q4.w;
  const double s = 2.0 / (((w * w + x * x) + y * y) + z * z);
  R[0] = 1.0 - s * (y * y + z * z);
  R[1] = s * (x * y - w * z);
  R[2] = s * (x * z + w * y);
  R[3] = s * (x * y + w * z);
  R[4] = 1.0 - s * (x * x + z * z);
  R[5] = s * (y * z - w * x);
  R[6] = s * (x * z - w * y);
  R[7] = s * (y * z + w * x);
  R[8] = 1.0 - s * (x * x + y * y);
}
__device__ __forceinline__ double3 mat_vec(const double* R, double3 v) {
  return dv((R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
            (R[6] * v.x + R[7] * v.y) + R[8] * v.z);
}
// v turned about the unit axis a by the angle of cosine c, sine s (FP64 Rodrigues)
__device__ __forceinline__ double3 rot_about_d(double3 a, double c, double s, double3 v) {
  const double3 axv = dcross(a, v);
  const double av = ddot(a, v);
  return dadd(dadd(dscale(v, c), dscale(axv, s)), dscale(a, av * (1.0 - c)));
}

// Closest point of triangle (a, b, c) to p (Ericson, Real-Time Collision
// Detection, 5.1.5), FP64.
__device__ __forceinline__ double3 closest_on_triangle_d(double3 p, double3 a, double3 b,
                                                         double3 c) {
  const double3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
  const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const double3 bp = dsub(p, b);
  const double d3_ = ddot(ab, bp), d4 = ddot(ac, bp);
  if (d3_ >= 0.0 && d4 <= d3_) return b;
  const double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) return dadd(a, dscale(ab, d1 / (d1 - d3_)));
  const double3 cp = dsub(p, c);
  const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return dadd(a, dscale(ac, d2 / (d2 - d6)));
  const double va = d3_ * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0)
    return dadd(b, dscale(dsub(c, b), (d4 - d3_) / ((d4 - d3_) + (d5 - d6))));
  const double den = 1.0 / ((va + vb) + vc);
  return dadd(dadd(a, dscale(ab, vb * den)), dscale(ac, vc * den));
}

// A contact of particle a with b (or a wall): unit normal n from b to a,
// overlap delta > 0, contact point relative to a's centre (ca) and to b's
// centre (cb).
struct MixHit {
  float3 n;
  float delta;
  float3 ca, cb;
};

// ------------------------------------------------------ sphere - polyhedron
// Sphere (centre c, radius r) against the polyhedron at x with world-frame
// geometry (V, F, faces, nf).  a = the sphere: n from the polyhedron to the
// sphere, ca = -r n, cb the nearest point of the hull (or the centre's
// projection on the deepest face when the centre is inside).
__device__ __forceinline__ bool sphere_hull(float3 c, float r, float3 x, const double4* V,
                                            const double4* F, const uchar4* faces, int nf,
                                            MixHit& h) {
  const double3 d = dsub(d3(c), d3(x));
  const double rr = (double)r;
  double smax = -1e300;
  int fb = 0;
  for (int f = 0; f < nf; ++f) {
    const double4 P = F[f];
    const double s = ((P.x * d.x + P.y * d.y) + P.z * d.z) - P.w;
    if (s > smax) { smax = s; fb = f; }
  }
  if (!(smax < rr)) return false;
  double3 q, nn;
  double delta;
  if (smax <= 0.0) {
    const double4 P = F[fb];
    nn = dxyz(P);
    delta = rr - smax;
    q = dsub(d, dscale(nn, smax));
  } else {
    double best = 1e300;
    q = d;
    for (int f = 0; f < nf; ++f) {
      const double4 P = F[f];
      const double s = ((P.x * d.x + P.y * d.y) + P.z * d.z) - P.w;
      if (!(s > 0.0 && s < rr)) continue;
      const uchar4 t = faces[f];
      const double3 qf = closest_on_triangle_d(d, dxyz(V[t.x]), dxyz(V[t.y]), dxyz(V[t.z]));
      const double3 e = dsub(d, qf);
      const double e2 = ddot(e, e);
      if (e2 < best) { best = e2; q = qf; }
    }
    if (!(best < rr * rr)) return false;
    const double dist = sqrt(best);
    if (!(dist > 0.0)) return false;
    nn = dv((d.x - q.x) / dist, (d.y - q.y) / dist, (d.z - q.z) / dist);
    delta = rr - dist;
  }
  const float df = (float)delta;
  if (!(df > 0.0f)) return false;
  h.n = to_f3(nn);
  h.delta = df;
  h.ca = h.n * (-r);
  h.cb = to_f3(q);
  return true;
}

// --------------------------------------------------- polyhedron pairs (SAT)
// Separation of hull B (vertex offsets VB, centre at d from A's centre) from
// the plane (unit normal, offset) P of a face of A.
__device__ __forceinline__ double face_sep(double4 P, double3 d, const double4* VB, int nvB) {
  double m = 1e300;
  for (int k = 0; k < nvB; ++k) {
    const double4 v = VB[k];
    const double t = (P.x * (d.x + v.x) + P.y * (d.y + v.y)) + P.z * (d.z + v.z);
    if (t < m) m = t;
  }
  return m - P.w;
}

constexpr double kNoAxis = -1e300;

// Edge ea = (PA, QA) of A with face normals (a, b), edge eb = (PB, QB) of B
// with face normals (c, dn), all relative to A's centre: when the arcs
// (a, b) and (-c, -dn) cross on the unit sphere (the edges form a face of
// the Minkowski difference), the separation along their cross product
// oriented away from A's centre, else kNoAxis.
__device__ __forceinline__ double edge_sep(double3 a, double3 b, double3 c, double3 dn, double3 PA,
                                           double3 QA, double3 PB, double3 QB) {
  c = dneg(c);
  dn = dneg(dn);
  const double3 bxa = dcross(b, a), dxc = dcross(dn, c);
  const double cba = ddot(c, bxa), dba = ddot(dn, bxa), adc = ddot(a, dxc), bdc = ddot(b, dxc);
  if (!(cba * dba < 0.0 && adc * bdc < 0.0 && cba * bdc > 0.0)) return kNoAxis;
  const double3 ea = dsub(QA, PA), eb = dsub(QB, PB);
  double3 ax = dcross(ea, eb);
  const double l2 = ddot(ax, ax);
  if (!(l2 > 1e-10 * (ddot(ea, ea) * ddot(eb, eb)))) return kNoAxis;   // parallel edges
  const double l = sqrt(l2);
  ax = dv(ax.x / l, ax.y / l, ax.z / l);
  if (ddot(ax, PA) < 0.0) ax = dneg(ax);
  return ddot(ax, dsub(PB, PA));
}

__device__ __forceinline__ double3 edge_axis(double3 PA, double3 QA, double3 PB, double3 QB) {
  const double3 ea = dsub(QA, PA), eb = dsub(QB, PB);
  double3 ax = dcross(ea, eb);
  const double l = sqrt(ddot(ax, ax));
  ax = dv(ax.x / l, ax.y / l, ax.z / l);
  if (ddot(ax, PA) < 0.0) ax = dneg(ax);
  return ax;
}

// Closest points of segments (P1, Q1) and (P2, Q2), not parallel (Ericson 5.1.9).
__device__ __forceinline__ double3 segments_midpoint(double3 P1, double3 Q1, double3 P2,
                                                     double3 Q2) {
  const double3 d1 = dsub(Q1, P1), d2 = dsub(Q2, P2), r = dsub(P1, P2);
  const double a = ddot(d1, d1), e = ddot(d2, d2), f = ddot(d2, r);
  const double c = ddot(d1, r), b = ddot(d1, d2);
  const double den = a * e - b * b;
  double s = den > 0.0 ? (b * f - c * e) / den : 0.0;
  s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  double t = (b * s + f) / e;
  if (t < 0.0) {
    t = 0.0;
    s = -c / a;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  } else if (t > 1.0) {
    t = 1.0;
    s = (b - c) / a;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  }
  const double3 c1 = dadd(P1, dscale(d1, s)), c2 = dadd(P2, dscale(d2, t));
  return dscale(dadd(c1, c2), 0.5);
}

// Feature tolerances of the pick between the queries (separations are <= 0
// when the hulls overlap): a face of B wins over a face of A only when its
// separation exceeds kMixRelFace times A's, an edge pair over the faces only
// when its separation exceeds kMixRelEdge times theirs.
constexpr double kMixRelFace = 0.98;
constexpr double kMixRelEdge = 0.90;

struct SatPick {
  double sA, sB, sE;
  int fA, fB, eE;
};

// 0: face of A, 1: face of B, 2: edge pair.
__device__ __forceinline__ int sat_kind(const SatPick& q) {
  const double sf = q.sA > q.sB ? q.sA : q.sB;
  if (q.sE > kMixRelEdge * sf) return 2;
  if (q.sB > kMixRelFace * q.sA) return 1;
  return 0;
}

// The contact from the picked axis: a = A (lower id), b = B; n from B to A,
// ca relative to A's centre, cb to B's (d = B's centre - A's).
__device__ __forceinline__ bool hull_hull_finish(const SatPick& q, double3 d, const double4* VA,
                                                 const double4* FA, const uchar4* EA, int nvA,
                                                 const double4* VB, const double4* FB,
                                                 const uchar4* EB, int nvB, int neB,
                                                 MixHit& h) {
  const int kind = sat_kind(q);
  double3 nAB, cp;
  double s;
  if (kind == 0) {
    const double4 P = FA[q.fA];
    nAB = dxyz(P);
    s = q.sA;
    double3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < nvB; ++k) {
      const double3 v = dadd(d, dxyz(VB[k]));
      const double t = ((P.x * v.x + P.y * v.y) + P.z * v.z) - P.w;
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else if (kind == 1) {
    const double4 P = FB[q.fB];
    nAB = dneg(dxyz(P));
    s = q.sB;
    double3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < nvA; ++k) {
      const double3 v = dxyz(VA[k]);
      const double3 w = dsub(v, d);
      const double t = ((P.x * w.x + P.y * w.y) + P.z * w.z) - P.w;
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else {
    const uchar4 ea = EA[q.eE / neB], eb = EB[q.eE % neB];
    const double3 PA = dxyz(VA[ea.x]), QA = dxyz(VA[ea.y]);
    const double3 PB = dadd(d, dxyz(VB[eb.x])), QB = dadd(d, dxyz(VB[eb.y]));
    nAB = edge_axis(PA, QA, PB, QB);
    s = q.sE;
    cp = segments_midpoint(PA, QA, PB, QB);
  }
  const float df = (float)(-s);
  if (!(df > 0.0f)) return false;
  h.n = to_f3(dneg(nAB));
  h.delta = df;
  h.ca = to_f3(cp);
  h.cb = to_f3(dsub(cp, d));
  return true;
}

// --------------------------------------------- polyhedron - triangle (SAT)
// Edge t of a triangle (t0, t1, t2): 0 = (t0, t1), 1 = (t0, t2), 2 = (t1, t2).
__device__ __forceinline__ int tri_e0(int t) { return t == 2 ? 1 : 0; }
__device__ __forceinline__ int tri_e1(int t) { return t == 0 ? 1 : 2; }

// The contact of hull_tri from its queries' results: the triangle's face
// (sT, tplus: +nt or -nt), the polyhedron's face (sP, fP), the edge pair
// (sE, eE = 3 edge + triangle edge, or -1; eplus: the triangle on the + side
// of the pair's axis).
__device__ __forceinline__ bool hull_tri_finish(const double4* V, const double4* F,
                                                const uchar4* E, int nv, const double3* T,
                                                double3 nt, double sT, bool tplus, double sP,
                                                int fP, double sE, int eE, bool eplus, MixHit& h,
                                                double3& nd, int& kind_out) {
  SatPick q;
  q.sA = sT;   // the wall's face plays the reference face
  q.sB = sP;
  q.sE = eE >= 0 ? sE : kNoAxis;
  const int kind = sat_kind(q);
  double3 n_in, cp;   // n_in: from the triangle to the polyhedron
  double s;
  if (kind == 0) {
    n_in = tplus ? nt : dneg(nt);
    s = sT;
    double3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < nv; ++k) {
      const double3 v = dxyz(V[k]);
      const double t = ddot(n_in, v) - ddot(n_in, T[0]);
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else if (kind == 1) {
    const double4 P = F[fP];
    n_in = dneg(dxyz(P));
    s = sP;
    double3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double t = ((P.x * T[k].x + P.y * T[k].y) + P.z * T[k].z) - P.w;
      if (t < 0.0) { acc = dadd(acc, dscale(T[k], -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else {
    const int e = eE / 3, t = eE % 3;
    const uchar4 ed = E[e];
    const double3 P0 = dxyz(V[ed.x]), Q0 = dxyz(V[ed.y]);
    const double3 P1 = T[tri_e0(t)], Q1 = T[tri_e1(t)];
    double3 ax = dcross(dsub(Q0, P0), dsub(Q1, P1));
    const double l = sqrt(ddot(ax, ax));
    ax = dv(ax.x / l, ax.y / l, ax.z / l);
    n_in = eplus ? dneg(ax) : ax;
    s = sE;
    cp = segments_midpoint(P0, Q0, P1, Q1);
  }
  const float df = (float)(-s);
  if (!(df > 0.0f)) return false;
  nd = n_in;
  kind_out = kind;
  h.n = to_f3(n_in);
  h.delta = df;
  h.ca = to_f3(cp);
  h.cb = h.ca;
  return true;
}

// Separation of the triangle T from the polyhedron's face plane P.
__device__ __forceinline__ double tri_face_sep(double4 P, const double3* T) {
  double m = 1e300;
  for (int k = 0; k < 3; ++k) {
    const double t = (P.x * T[k].x + P.y * T[k].y) + P.z * T[k].z;
    if (t < m) m = t;
  }
  return m - P.w;
}

// Separation along the triangle's normal nt or -nt (the larger; tplus: +nt)
// from the polyhedron's extent [lo, hi] along nt.
__device__ __forceinline__ double tri_plane_sep(double3 nt, const double3* T, double lo,
                                                double hi, bool& tplus) {
  const double h0 = ddot(nt, T[0]);
  const double sTp = lo - h0, sTm = h0 - hi;
  tplus = sTp >= sTm;
  return tplus ? sTp : sTm;
}

// Edge pair x = 3 e + t (edge e of the polyhedron, edge t of the triangle):
// the separation along their cross product with full support extents of
// both (plus: the triangle on the + side), kNoAxis for parallel edges.
__device__ __forceinline__ double tri_edge_sep(const double4* V, const uchar4* E, int nv,
                                               const double3* T, int x, bool& plus) {
  const int e = x / 3, t = x % 3;
  const uchar4 ed = E[e];
  const double3 P0 = dxyz(V[ed.x]), ep = dsub(dxyz(V[ed.y]), P0);
  const double3 et = dsub(T[tri_e1(t)], T[tri_e0(t)]);
  double3 ax = dcross(ep, et);
  const double l2 = ddot(ax, ax);
  if (!(l2 > 1e-10 * (ddot(ep, ep) * ddot(et, et)))) return kNoAxis;
  const double l = sqrt(l2);
  ax = dv(ax.x / l, ax.y / l, ax.z / l);
  double pmin = 1e300, pmax = -1e300;
  for (int k = 0; k < nv; ++k) {
    const double u = ddot(ax, dxyz(V[k]));
    if (u < pmin) pmin = u;
    if (u > pmax) pmax = u;
  }
  double tmin = 1e300, tmax = -1e300;
  for (int k = 0; k < 3; ++k) {
    const double u = ddot(ax, T[k]);
    if (u < tmin) tmin = u;
    if (u > tmax) tmax = u;
  }
  const double s1 = tmin - pmax, s2 = pmin - tmax;
  plus = s1 >= s2;
  return plus ? s1 : s2;
}

// The triangle T (vertices relative to the polyhedron's centre, unit normal
// nt) as a flat hull against the polyhedron (V, F, E; its faces' normals
// outward).  a = the polyhedron: n from the triangle to it, ca relative to
// its centre.  Returns the kind of axis through `kind` (0 the triangle's
// face, 1 a face of the polyhedron, 2 an edge pair) and the unrounded
// normal through `nd`, for the choice among a polyhedron's triangle
// contacts.
__device__ __forceinline__ bool hull_tri(const double4* V, const double4* F, const uchar4* E,
                                         int nv, int nf, int ne, const double3* T, double3 nt,
                                         MixHit& h, double3& nd, int& kind) {
  double sP = -1e300;
  int fP = 0;
  for (int f = 0; f < nf; ++f) {
    const double s = tri_face_sep(F[f], T);
    if (s > sP) { sP = s; fP = f; }
  }
  if (sP > 0.0) return false;
  double lo = 1e300, hi = -1e300;
  for (int k = 0; k < nv; ++k) {
    const double t = ddot(nt, dxyz(V[k]));
    if (t < lo) lo = t;
    if (t > hi) hi = t;
  }
  bool tplus;
  const double sT = tri_plane_sep(nt, T, lo, hi, tplus);
  if (sT > 0.0) return false;
  double sE = -1e300;
  int eE = -1;
  bool eplus = true;
  for (int x = 0; x < 3 * ne; ++x) {
    bool pl;
    const double s = tri_edge_sep(V, E, nv, T, x, pl);
    if (s == kNoAxis) continue;
    if (s > 0.0) return false;
    if (s > sE) { sE = s; eE = x; eplus = pl; }
  }
  return hull_tri_finish(V, F, E, nv, T, nt, sT, tplus, sP, fP, sE, eE, eplus, h, nd, kind);
}

// ----------------------------------------------------- polyhedron - plane
// Plane n . x = pd (n into the domain) against the polyhedron at x: the
// deepest vertex's depth, the vertices below the plane weighted by depth.
__device__ __forceinline__ bool hull_plane(float3 n, float pd, float3 x, const double4* V, int nv,
                                           MixHit& h) {
  const double3 nn = d3(n);
  const double base = ddot(nn, d3(x)) - (double)pd;
  double lo = 1e300, wsum = 0.0;
  double3 acc = dv(0.0, 0.0, 0.0);
  for (int k = 0; k < nv; ++k) {
    const double3 v = dxyz(V[k]);
    const double s = base + ddot(nn, v);
    if (s < lo) lo = s;
    if (s < 0.0) { acc = dadd(acc, dscale(v, -s)); wsum = wsum - s; }
  }
  const float df = (float)(-lo);
  if (!(df > 0.0f) || !(wsum > 0.0)) return false;
  h.n = n;
  h.delta = df;
  h.ca = to_f3(dscale(acc, 1.0 / wsum));
  h.cb = h.ca;
  return true;
}

// Coplanar wall contacts (a polyhedron over two triangles of one plane):
// only the deepest of them counts.
constexpr double kMixCoplanar = 1.0 - 1e-9;

// ---------------------------------------------------------------- the laws
// Contact h of particle a (mass ma, velocity va, spin wa) with particle b:
// the linear law with tangential history on the contact point's relative
// velocity (no rolling friction); the force on a and the torques on a and b
// about their centres.  Both particles' steps evaluate it with the same
// arguments (a the sphere of a sphere-polyhedron pair, the lower id of two
// polyhedra), so the pair's forces cancel bit for bit.
__device__ __forceinline__ void mix_pair_law(const EnsSysDev& S, const MixHit& h, float ma,
                                             float3 va, float3 wa, float mb, float3 vb,
                                             float3 wb, float dt, float3& xi, float3& F,
                                             float3& Ta, float3& Tb) {
  const float3 vct = (va + cross3(wa, h.ca)) - (vb + cross3(wb, h.cb));
  const float ms = (ma * mb) / (ma + mb);
  float3 t0;
  contact_law<kLawLinear, false>(S, S.mu, h.n, h.delta, 0.0f, ms, vct, vct,
                                 f3(0.0f, 0.0f, 0.0f), 0.0f, dt, xi, F, t0);
  Ta = cross3(h.ca, F);
  Tb = cross3(h.cb, f3(-F.x, -F.y, -F.z));
}

// A polyhedron (a) against a wall moving at vw at the contact point.
__device__ __forceinline__ void mix_wall_law(const EnsSysDev& S, const MixHit& h, float ma,
                                             float3 va, float3 wa, float3 vw, float dt,
                                             float3& xi, float3& F, float3& Ta) {
  const float3 vct = (va + cross3(wa, h.ca)) - vw;
  float3 t0;
  contact_law<kLawLinear, false>(S, S.mu_w, h.n, h.delta, 0.0f, ma, vct, vct,
                                 f3(0.0f, 0.0f, 0.0f), 0.0f, dt, xi, F, t0);
  Ta = cross3(h.ca, F);
}

}  // namespace blaze
