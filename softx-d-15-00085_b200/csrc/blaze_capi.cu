// blaze_capi.cu -- host side of libblaze_b200.so: one simulation object per
// handle (device buffers allocated once, a private CUDA stream), the step
// pipeline, and the C ABI of include/blaze_dem.h.
//
// The reference allocates and frees its sort temporaries and contact list
// inside every step and synchronises after every stage
// (DeviceInterface.cu:1825-2513); here every buffer lives for the whole run
// and a step is a fixed sequence of kernel launches on one stream.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "blaze_dem.h"
#include "dem_kernels.cuh"
#include "poly_kernels.cuh"
#include "radix_sort.cuh"

using namespace blaze;

#define CK(x)                                  \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_); \
  } while (0)

namespace {

int cuda_fail(cudaError_t e) {
  std::fprintf(stderr, "blaze: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
  return -(1000 + (int)e);
}

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

}  // namespace

struct blaze_sim {
  int n_max = 0;
  SimulationInfo si{};
  WOBJ w[8]{};
  POBJ p[8]{};
  DOBJ d[kMaxDobj]{};
  int n_w = 0, n_p = 0, n_d = 0;
  int num_wobj = 0;
  blaze_options opt{};
  int cyl_rot = 0;
  SimParams hp{};
  SimParams* dp = nullptr;
  std::vector<WallOp> ops;
  WallOp* d_ops = nullptr;
  uint32_t* d_wall_off = nullptr;
  uint16_t* d_wall_idx = nullptr;
  bool walls_static = true;
  // state
  StateBuf S[3]{};  // S[0], S[1] ping-pong, S[2] sorted gather target
  OrderBuf ob{};
  int cur = 0;      // S[cur] holds the current state
  RadixSortBuffers rs{};
  uint32_t* cstart = nullptr;
  uint32_t* cend = nullptr;
  NbrList nl{};
  StepCtl* ctl = nullptr;
  StepCtl* h_ctl = nullptr;  // pinned mirror
  ForceCapture cap{};
  bool cap_alloc = false;
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;          // captures conditional bodies
  cudaStream_t aux2 = nullptr;         // captures the IF bodies nested in a SWITCH body
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // kGraphSteps steps, starting at cur = 0 / 1
  // with a skin: a block of kGraphSteps steps whose kind the device picks
  // (build_block), per start; and one step as a graph, per start, per
  // (block start, check after the step) (build_single)
  cudaGraphExec_t block[2] = {nullptr, nullptr};
  cudaGraphExec_t single[2][2][2] = {};
  int step_launches = 0;               // kernels of one step, counted when a graph is built
  int* d_rb = nullptr;                 // per graph step: nonzero when that step re-sorted
  uint32_t* d_chk = nullptr;           // list-check maxima slots (StepCtl::chk)
  bool spin_free = false;              // rotation off and every angular velocity zero
  int key_bits = 1;
  uint32_t cells_cap = 0;   // entries allocated in cstart / cend
  long long steps = 0;
  // with a skin, steps below this index each end with a list check (from a
  // forced re-sort to the next multiple of kListCheckEvery; see force_check)
  long long check_until = 0;
  int stepc = 0;        // steps since the last removal check
  uint32_t status = 0;  // accumulated, reported at sync points
  int last_launches = 0;
  // energy tallies (SimulationInfo::EnergyCalc): particle-particle, volume
  // objects, world objects, FP64 on the device; per-particle values of the
  // step and per-block partial sums when the step computes them
  double* d_tally = nullptr;
  double* d_eb = nullptr;
  double* d_epart = nullptr;
  float fc = 0.0f;
  // the mill driver's per-step moves on the device (blaze_set_dobj_rotation,
  // blaze_set_dobj_translation, blaze_set_wobj_rotation); the device copies
  // of the objects are then the current ones
  bool dobj_rot = false;
  int dobj_tr = -1;
  bool dobj_on_device = false;
  float rot_ax = 0.0f, rot_ay = 0.0f, rot_c = 1.0f, rot_s = 0.0f, rot_rad = 0.0f;
  // the mill's fill waves (InitConfig grid_type 2): fill_pack particles join
  // the run every fill_clear + 1 steps until all are in
  bool filling = false;
  int fill_n = 0, fill_pack = 0, fill_clear = 0, fill_counter = 0;
  bool wobj_rot = false;
  bool wobj_on_device = false;
  uint32_t wrot_mask = 0;
  float wrot_ax = 0.0f, wrot_ay = 0.0f, wrot_c = 1.0f, wrot_s = 0.0f, wrot_rad = 0.0f;
  // optional per-phase event timing (non-graph stepping only)
  bool profile = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_marks;  // (phase, event index) start/end pairs in order
  int ev_used = 0;
  // device staging of the reference interface's AoS host arrays (n_max
  // each), packed / unpacked by a kernel, and its two result words (pinned)
  HostStage stage{};
  int* h_flags = nullptr;
  unsigned int* d_count = nullptr;     // blaze_count_above's device word
  // convex polyhedra (particle_type 1): body-frame objects and the
  // world-frame geometry the step rebuilds
  bool poly = false;
  PolyShape* d_shapes = nullptr;
  PolyGeom geom{};
  PolyPairs pairs{};
};

namespace {

constexpr int kGraphSteps = kListCheckEvery;
blaze_sim* g_default = nullptr;

void drop_graphs(blaze_sim* s);

// ------------------------------------------------------------------ params
void build_params(blaze_sim* s) {
  SimParams& P = s->hp;
  std::memset(&P, 0, sizeof(P));
  const SimulationInfo& si = s->si;
  P.origin = si.worldOrigin;
  P.cell = si.cellSize;
  P.ncells = si.num_NNCells;
  if (s->opt.skin > 0.0f) {
    // A Verlet list keeps pairs up to ra + rb + skin apart, and the 27-cell
    // search finds a pair only when it lies within one cell edge: the list
    // grid's cells are at least 2 r_max + skin, over the project grid's
    // extent (the project's cells, 2 r_max in the shipped worlds, serve the
    // contacts-only search of reference mode).
    float rmax = 0.0f;
    for (int t = 0; t < s->n_p; ++t) rmax = std::max(rmax, s->p[t].radius);
    const float need = 2.0f * rmax + s->opt.skin;
    float* c[3] = {&P.cell.x, &P.cell.y, &P.cell.z};
    int* nc[3] = {&P.ncells.x, &P.ncells.y, &P.ncells.z};
    for (int a = 0; a < 3; ++a) {
      if (*c[a] >= need) continue;
      const double extent = (double)*nc[a] * (double)*c[a];
      *c[a] = need;
      *nc[a] = std::max(1, (int)std::ceil(extent / (double)need));
    }
  }
  const long long nx = P.ncells.x, ny = P.ncells.y, nz = P.ncells.z;
  const long long hmax = (nx - 1) + (nz - 1) * nz + (ny - 1) * nx * nz + 1;
  const long long prod = nx * ny * nz;
  P.ncell_tab = (uint32_t)std::max(hmax, prod);
  P.gravity = si.Force_Field;
  P.dt = si.InitalDelta_t;
  P.tan_k = si.InitalDelta_t > 0.0f ? 0.025f / si.InitalDelta_t : 0.0f;
  P.roll_res = si.Roll_Res;
  P.mill_rot_vel = si.MillRotVel;
  P.drum_r = s->n_w > 0 ? s->w[0].cyl_geo.radius : 0.0f;
  P.rotation = si.Rotation ? 1 : 0;
  P.mode2d = si.Mode2D ? 1 : 0;
  P.energy_calc = si.EnergyCalc ? 1 : 0;
  P.is_mill = si.isMillSim ? 1 : 0;
  P.rotating_wobj = si.Rotating_WObject ? 1 : 0;
  P.cyl_rot = s->cyl_rot;
  P.cent = si.cent;
  P.dobj_cyl_bound_r = si.DObject_CylinderBoundR;
  P.n_types = s->n_p;
  for (int t = 0; t < s->n_p; ++t) {
    const POBJ& o = s->p[t];
    TypeParams& T = P.types[t];
    T.radius = o.radius;
    T.mass = o.mass;
    T.iinv = o.InertiaT[0];
    T.com = o.COM;
    T.s_kn = o.surface_Kn; T.s_cn = o.surface_Cn;
    T.s_mus = o.surface_Fric_static; T.s_muk = o.surface_Fric_kinetic;
    T.d_kn = o.Dsurface_Kn; T.d_cn = o.Dsurface_Cn; T.d_muk = o.Dsurface_Fric_kinetic;
    for (int q = 0; q < kMaxPP; ++q) T.pp[q] = o.PP[q];
  }
  P.n_dobj = s->n_d;
  for (int k = 0; k < s->n_d; ++k) {
    const DOBJ& D = s->d[k];
    DobjDev& G = P.dobj[k];
    G.com = D.COM;
    G.axis = D.Axis;
    G.bound_r = D.boundR;
    G.num_faces = std::min(D.num_faces, 3);
    G.num_edges = std::min(D.num_edges, 4);
    G.num_vertex = std::min(std::max(D.num_vertex, 0), 8);
    G.attached = D.is_attached_DWorld ? 1 : 0;
    G.translating = D.is_translating ? 1 : 0;
    G.velocity = D.velocity;
    for (int v = 0; v < 8; ++v) G.vert[v] = D.vertex[v];
    for (int f = 0; f < 3; ++f) G.faces[f] = D.faces[f];
    for (int e = 0; e < 4; ++e) {
      G.edge0[e] = (int)(D.edge[e].point_vindex[0] & 7u);
      G.edge1[e] = (int)(D.edge[e].point_vindex[1] & 7u);
    }
  }
  P.max_nbr = s->opt.max_nbr;
  P.skin = s->opt.skin;
}

// World objects -> the wall program, in world-object order
// (DEM_Kernels_Compute.cuh:312-600).
void build_ops(blaze_sim* s) {
  s->ops.clear();
  for (int k = 0; k < s->num_wobj && k < s->n_w; ++k) {
    const WOBJ& W = s->w[k];
    if (W.surface_type == plane) {
      for (int f = 0; f < W.num_surfaces && f < 16; ++f) {
        const Surface& S = W.surfaces[f];
        WallOp op;
        std::memset(&op, 0, sizeof(op));
        op.kind = S.area == -1.0f ? kOpPlane : kOpFace;
        op.wobj = k;
        op.nv = std::min(std::max(S.num_vertex, 0), 8);
        op.area = S.area;
        op.tol = S.Tol;
        op.n = S.normal;
        op.c = S.centroid;
        for (int v = 0; v < op.nv; ++v) op.v[v] = W.vertex[S.vertex_Order[v] & 15];
        s->ops.push_back(op);
      }
    } else if (W.surface_type == cylinder) {
      const Macro_Cylinder& cg = W.cyl_geo;
      WallOp op;
      std::memset(&op, 0, sizeof(op));
      op.kind = kOpCylinder;
      op.wobj = k;
      op.radius = cg.radius;
      op.axis = cg.AXIS;
      op.cbot = cg.center_bot_cap;
      s->ops.push_back(op);
      if (cg.has_top_cap) {
        WallOp t = op;
        t.kind = kOpCapTop;
        t.n = cg.normal_top_cap;
        t.c = cg.center_top_cap;
        s->ops.push_back(t);
      }
      if (cg.has_bot_cap) {
        WallOp b = op;
        b.kind = kOpCapBot;
        b.n = cg.normal_bot_cap;
        b.c = cg.center_bot_cap;
        s->ops.push_back(b);
      }
    }
  }
  s->hp.n_ops = (int)s->ops.size();
}

// Per-cell candidate lists of wall ops, conservative: an op is dropped for a
// cell only when no sphere centred in that cell (radius <= rmax) can pass
// the op's contact test, so the forces are unchanged bit for bit.  Over the
// eight corners of the cell (the tests are affine or convex in the centre):
//   faces, planes, caps: contact needs n.(x - c) in (0, r); kept when the
//            corner range of n.(x - c) meets (-eps, rmax + eps); faces also
//            need the centre to project inside the polygon grown by the
//            area tolerance (is_PointOnSurface accepts a point at distance d
//            outside a convex polygon of area A while d * L <= Tol/100 * A
//            for the edge length L nearest to it; the margin uses the
//            shortest edge), tested as a box overlap
//   cylinder: contact needs |x*AXIS - c_bot| + r > R; kept when the
//            farthest corner reaches R - rmax - eps.
void build_wall_grid(blaze_sim* s, std::vector<uint32_t>& off, std::vector<uint16_t>& idx) {
  const SimParams& P = s->hp;
  const uint32_t nt = P.ncell_tab;
  float rmax = 0.0f;
  for (int t = 0; t < s->n_p; ++t) rmax = std::max(rmax, s->p[t].radius);
  const double eps = 1e-3;
  struct Box { double lo[3], hi[3]; };
  const int nops = (int)s->ops.size();
  std::vector<Box> grown(nops);
  std::vector<int> always(nops, 0);
  for (int q = 0; q < nops; ++q) {
    const WallOp& op = s->ops[q];
    if (op.kind != kOpFace) continue;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    double minedge = 1e300;
    for (int v = 0; v < op.nv; ++v) {
      const float3 a = op.v[v], b = op.v[(v + 1) % op.nv];
      const double ax[3] = {a.x, a.y, a.z};
      for (int c = 0; c < 3; ++c) { lo[c] = std::min(lo[c], ax[c]); hi[c] = std::max(hi[c], ax[c]); }
      const double e = std::sqrt((double)(a.x - b.x) * (a.x - b.x) + (double)(a.y - b.y) * (a.y - b.y) +
                                 (double)(a.z - b.z) * (a.z - b.z));
      if (e > 0) minedge = std::min(minedge, e);
    }
    double margin = (double)op.tol / 100.0 * std::fabs((double)op.area) / std::max(minedge, 1e-12);
    margin = margin * 1.01 + 1e-4 * (hi[0] - lo[0] + hi[1] - lo[1] + hi[2] - lo[2]) + rmax + eps;
    if (!std::isfinite(margin) || !(op.area > 0.0f) || op.nv < 3) { always[q] = 1; continue; }
    for (int c = 0; c < 3; ++c) { grown[q].lo[c] = lo[c] - margin; grown[q].hi[c] = hi[c] + margin; }
  }
  off.assign((size_t)nt + 1, 0);
  idx.clear();
  const int3 nc = P.ncells;
  // hashes alias when ncx != ncz: a hash's list is the union over its cells
  std::vector<std::vector<uint16_t>> by_hash((size_t)nt);
  for (int gy = 0; gy < nc.y; ++gy)
    for (int gz = 0; gz < nc.z; ++gz)
      for (int gx = 0; gx < nc.x; ++gx) {
        const uint32_t h = (uint32_t)((gx + gz * nc.z) + (gy * nc.x) * nc.z);
        const double lo[3] = {P.origin.x + (double)gx * P.cell.x, P.origin.y + (double)gy * P.cell.y,
                              P.origin.z + (double)gz * P.cell.z};
        const double hi[3] = {lo[0] + P.cell.x, lo[1] + P.cell.y, lo[2] + P.cell.z};
        std::vector<uint16_t>& L = by_hash[h];
        for (int q = 0; q < nops; ++q) {
          const WallOp& op = s->ops[q];
          bool keep = always[q] != 0;
          if (!keep) {
            double dmin = 1e300, dmax = -1e300;
            for (int k = 0; k < 8; ++k) {
              const double x[3] = {(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
              if (op.kind == kOpCylinder) {
                const double px = x[0] * op.axis.x - op.cbot.x, py = x[1] * op.axis.y - op.cbot.y,
                             pz = x[2] * op.axis.z - op.cbot.z;
                dmax = std::max(dmax, std::sqrt(px * px + py * py + pz * pz));
              } else {
                const double d = (double)op.n.x * (x[0] - op.c.x) + (double)op.n.y * (x[1] - op.c.y) +
                                 (double)op.n.z * (x[2] - op.c.z);
                dmin = std::min(dmin, d);
                dmax = std::max(dmax, d);
              }
            }
            if (op.kind == kOpCylinder) {
              keep = dmax + rmax + eps > (double)op.radius;
            } else {
              keep = dmax > -eps && dmin < rmax + eps;
              if (keep && op.kind == kOpFace)
                for (int c = 0; c < 3; ++c)
                  if (hi[c] < grown[q].lo[c] || lo[c] > grown[q].hi[c]) keep = false;
            }
          }
          if (keep && std::find(L.begin(), L.end(), (uint16_t)q) == L.end()) L.push_back((uint16_t)q);
        }
        if (L.size() > 1) std::sort(L.begin(), L.end());
      }
  for (uint32_t h = 0; h < nt; ++h) {
    off[h] = (uint32_t)idx.size();
    idx.insert(idx.end(), by_hash[h].begin(), by_hash[h].end());
  }
  off[nt] = (uint32_t)idx.size();
}

// With the volume objects turned on the device, copy them back into the
// host's DOBJ and parameter mirrors (vertices, faces, centre of mass) before
// anything re-uploads the parameters from the host.
int pull_dobj(blaze_sim* s) {
  if (!s->dobj_on_device) return 0;
  CK(cudaStreamSynchronize(s->stream));
  const char* src = reinterpret_cast<const char*>(s->dp) + offsetof(SimParams, dobj);
  CK(cudaMemcpy(s->hp.dobj, src, sizeof(DobjDev) * kMaxDobj, cudaMemcpyDeviceToHost));
  for (int k = 0; k < s->n_d; ++k) {
    const DobjDev& G = s->hp.dobj[k];
    DOBJ& D = s->d[k];
    for (int v = 0; v < G.num_vertex; ++v) D.vertex[v] = G.vert[v];
    for (int f = 0; f < G.num_faces; ++f) {
      D.faces[f].centroid = G.faces[f].centroid;
      D.faces[f].normal = G.faces[f].normal;
      D.faces[f].area = G.faces[f].area;
    }
    D.COM = G.com;
  }
  return 0;
}

// With the world objects turned on the device, copy the wall program back
// and write its faces into the host's WOBJ mirror (vertices through
// vertex_Order, normal, centroid, area), walking the objects in build_ops'
// order.
int pull_wobj(blaze_sim* s) {
  if (!s->wobj_on_device || s->ops.empty()) return 0;
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(s->ops.data(), s->d_ops, sizeof(WallOp) * s->ops.size(), cudaMemcpyDeviceToHost));
  size_t q = 0;
  for (int k = 0; k < s->num_wobj && k < s->n_w; ++k) {
    WOBJ& W = s->w[k];
    if (W.surface_type == plane) {
      for (int f = 0; f < W.num_surfaces && f < 16 && q < s->ops.size(); ++f, ++q) {
        const WallOp& op = s->ops[q];
        if (!W.is_rotating) continue;
        Surface& S = W.surfaces[f];
        for (int v = 0; v < op.nv; ++v) W.vertex[S.vertex_Order[v] & 15] = op.v[v];
        S.normal = op.n;
        S.centroid = op.c;
        S.area = op.area;
      }
    } else if (W.surface_type == cylinder) {
      q += 1 + (W.cyl_geo.has_top_cap ? 1 : 0) + (W.cyl_geo.has_bot_cap ? 1 : 0);
    }
  }
  return 0;
}

int upload_walls(blaze_sim* s) {
  int rc = pull_dobj(s);
  if (!rc) rc = pull_wobj(s);
  if (rc) return rc;
  drop_graphs(s);
  build_ops(s);
  CK(cudaMemcpyAsync(s->dp, &s->hp, sizeof(SimParams), cudaMemcpyHostToDevice, s->stream));
  if (s->d_ops) CK(cudaFree(s->d_ops));
  s->d_ops = nullptr;
  CK(dalloc(&s->d_ops, s->ops.size()));
  if (!s->ops.empty())
    CK(cudaMemcpyAsync(s->d_ops, s->ops.data(), sizeof(WallOp) * s->ops.size(),
                       cudaMemcpyHostToDevice, s->stream));
  if (s->d_wall_off) CK(cudaFree(s->d_wall_off));
  if (s->d_wall_idx) CK(cudaFree(s->d_wall_idx));
  s->d_wall_off = nullptr;
  s->d_wall_idx = nullptr;
  if (s->opt.wall_grid && s->walls_static && !s->ops.empty()) {
    std::vector<uint32_t> off;
    std::vector<uint16_t> idx;
    build_wall_grid(s, off, idx);
    CK(dalloc(&s->d_wall_off, off.size()));
    CK(dalloc(&s->d_wall_idx, idx.size()));
    CK(cudaMemcpyAsync(s->d_wall_off, off.data(), sizeof(uint32_t) * off.size(),
                       cudaMemcpyHostToDevice, s->stream));
    if (!idx.empty())
      CK(cudaMemcpyAsync(s->d_wall_idx, idx.data(), sizeof(uint16_t) * idx.size(),
                         cudaMemcpyHostToDevice, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int upload_params(blaze_sim* s) {
  int rc = pull_dobj(s);
  if (!rc) rc = pull_wobj(s);
  if (rc) return rc;
  build_params(s);
  return upload_walls(s);
}

// The cell table and the sort's key width for the current grid (the list
// grid with a skin, the project's without); reallocated when the grid grows.
int alloc_cells(blaze_sim* s) {
  const uint32_t nt = s->hp.ncell_tab;
  const uint32_t top = nt + 1u;
  s->key_bits = 1;
  while (s->key_bits < 32 && (top >> s->key_bits) != 0) s->key_bits++;
  if (nt > s->cells_cap) {
    if (s->cstart) CK(cudaFree(s->cstart));
    if (s->cend) CK(cudaFree(s->cend));
    s->cstart = s->cend = nullptr;
    s->cells_cap = 0;
    CK(dalloc(&s->cstart, nt));
    CK(dalloc(&s->cend, nt));
    s->cells_cap = nt;
  }
  CK(cudaMemset(s->cstart, 0xff, sizeof(uint32_t) * nt));
  CK(cudaMemset(s->cend, 0xff, sizeof(uint32_t) * nt));
  return 0;
}

// Per-slot narrow-phase buffers of the polyhedron passes, sized by the
// neighbour list (slots are indexed with 32 bits).
int alloc_poly_pairs(blaze_sim* s) {
  PolyPairs& pp = s->pairs;
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(pp.status); f(pp.hint); f(pp.con); f(pp.qv); f(pp.qe); f(pp.counts);
  pp = PolyPairs{};
  const size_t slots = (size_t)s->nl.cap * (size_t)s->nl.stride;
  if (slots >= (size_t)0xffffffffu) {
    std::fprintf(stderr, "blaze: %zu neighbour slots exceed the polyhedron passes' 32-bit index\n",
                 slots);
    return -1;
  }
  CK(dalloc(&pp.status, slots));
  CK(dalloc(&pp.hint, slots));
  CK(cudaMemset(pp.hint, 0xff, slots));
  CK(dalloc(&pp.con, 2 * slots));
  CK(dalloc(&pp.qv, slots));
  CK(dalloc(&pp.qe, slots));
  CK(dalloc(&pp.counts, 3));
  CK(cudaMemset(pp.counts, 0, 3 * sizeof(int)));
  // the contact-list kernel also lists every filled slot for the passes
  if (s->nl.flat) CK(cudaFree(s->nl.flat));
  CK(dalloc(&s->nl.flat, slots));
  s->nl.flat_n = pp.counts + 2;
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  pp.grid_s = 16 * sms;
  pp.grid_v = 8 * sms;
  pp.grid_e = 8 * sms;
  return 0;
}

int alloc_nlist(blaze_sim* s) {
  drop_graphs(s);
  if (s->nl.idx) CK(cudaFree(s->nl.idx));
  if (s->nl.cnt) CK(cudaFree(s->nl.cnt));
  if (s->nl.flat) CK(cudaFree(s->nl.flat));
  s->nl.flat = nullptr;
  s->nl.flat_n = nullptr;
  s->nl.stride = s->n_max;
  s->nl.cap = s->opt.max_nbr;
  CK(dalloc(&s->nl.idx, (size_t)s->n_max * s->nl.cap));
  CK(dalloc(&s->nl.cnt, s->n_max));
  CK(cudaMemsetAsync(s->nl.cnt, 0, sizeof(uint32_t) * s->n_max, s->stream));
  if (s->poly) return alloc_poly_pairs(s);
  return 0;
}

int alloc_capture(blaze_sim* s) {
  if (s->cap_alloc || !s->opt.capture_forces) return 0;
  drop_graphs(s);
  float** ps[6] = {&s->cap.f_pp, &s->cap.t_pp, &s->cap.f_w, &s->cap.t_w, &s->cap.f_l, &s->cap.t_l};
  for (auto* q : ps) {
    CK(dalloc(q, (size_t)3 * s->n_max));
    CK(cudaMemsetAsync(*q, 0, sizeof(float) * 3 * s->n_max, s->stream));
  }
  s->cap_alloc = true;
  return 0;
}

// --------------------------------------------------------------- the step
int enqueue_rebuild(blaze_sim* s, const int* gate, cudaStream_t st) {
  const int n = s->n_max;
  launch_hash(s->dp, s->S[s->cur], s->ob, n, s->rs.keys[0], s->ctl, gate, st);
  const int res = radix_sort_pairs(s->rs, n, s->key_bits, true, gate, st);
  const size_t cbytes = sizeof(uint32_t) * s->hp.ncell_tab;
  CK(cudaMemsetAsync(s->cstart, 0xff, cbytes, st));
  launch_reorder(s->S[s->cur], s->S[2], s->ob, n, s->rs.keys[res], s->rs.vals[res], s->cstart,
                 s->cend, s->hp.ncell_tab, s->n_d > 0, s->nl.flat_n, s->ctl, gate, st);
  launch_nlist(s->dp, s->S[2], n, s->cstart, s->cend, s->nl, s->ctl, gate, st);
  s->last_launches += 3 + 3 * std::max(1, (s->key_bits + kRadixBits - 1) / kRadixBits);
  return 0;
}

cudaEvent_t prof_event(blaze_sim* s, int phase) {
  if ((int)s->ev_pool.size() <= s->ev_used) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    s->ev_pool.push_back(e);
  }
  cudaEvent_t e = s->ev_pool[s->ev_used];
  s->ev_marks.push_back({phase, s->ev_used});
  s->ev_used++;
  cudaEventRecord(e, s->stream);
  return e;
}

// The kernels of one step after the (conditional) re-sort, reading S[cur]
// or the sorted copy S[2] as `link` says and writing S[cur ^ 1]; returns the
// number of launches.
int enqueue_step_kernels(blaze_sim* s, StepLink link, cudaStream_t st) {
  const ForceCapture* cap = s->opt.capture_forces ? &s->cap : nullptr;
  int k = 1;
  if (s->dobj_rot || s->dobj_tr >= 0) {
    launch_move_dobj(s->dp, s->dobj_rot ? 1 : 0, s->rot_ax, s->rot_ay, s->rot_c, s->rot_s,
                     s->dobj_tr, s->n_d, st);
    ++k;
  }
  if (s->wobj_rot) {
    launch_rotate_wobj(s->d_ops, (int)s->ops.size(), s->wrot_mask, s->wrot_ax, s->wrot_ay,
                       s->wrot_c, s->wrot_s, st);
    ++k;
  }
  double* eb = s->hp.energy_calc ? s->d_eb : nullptr;   // allocated when EnergyCalc
  if (s->poly) {
    launch_poly_geom(s->d_shapes, s->geom, s->S[s->cur], s->S[2], s->ob, s->n_max,
                     s->si.Rotation ? 1 : 0, s->ctl, link.rebuilt, st);
    const int np = launch_poly_pairs(s->dp, s->d_shapes, s->geom, s->S[s->cur], s->S[2],
                                     s->n_max, s->nl, s->ctl, link.rebuilt, s->pairs, st);
    launch_poly_step(s->dp, s->d_shapes, s->geom, s->d_ops, s->S[s->cur], s->S[2],
                     s->S[s->cur ^ 1], s->ob, s->n_max, s->nl, s->pairs, s->ctl, link, cap, eb,
                     st);
    k += 1 + np;
  } else {
    launch_step(s->dp, s->d_ops, WallGrid{s->d_wall_off, s->d_wall_idx}, s->S[s->cur], s->S[2],
                s->S[s->cur ^ 1], s->ob, s->n_max, s->nl, s->ctl, link, s->spin_free, cap, eb,
                s->opt.fast_law != 0, st);
  }
  if (eb) {
    launch_energy_reduce(eb, s->n_max, s->ctl, s->d_epart, s->d_tally, st);
    k += 2;
  }
  return k;
}

// the list check's look-ahead distance per unit speed (list_needs_rebuild)
float list_look(const blaze_sim* s) { return 2.0f * kListCheckEvery * s->si.InitalDelta_t; }

// The largest surface speed of a moving wall or volume object, cm/s (0 when
// all are at rest): the drum wall turning at MillRotVel (cylinder rotation,
// and the faces of a rotating world object under it), volume objects
// attached to a mill drum (they meet particles at the drum's wall velocity,
// DEM_Kernels_Compute.cuh:206-216), lifters turned on the device, a
// translating volume object, world objects turned on the device.  The list
// check counts it as a particle speed at every block start: a moving wall
// can set a particle at rest in motion within the block.
float wall_speed(const blaze_sim* s) {
  const float dt = s->si.InitalDelta_t;
  auto rxy = [](float3 p, float ax, float ay) {
    return std::sqrt((p.x - ax) * (p.x - ax) + (p.y - ay) * (p.y - ay));
  };
  const float om_drum = std::fabs(s->hp.mill_rot_vel);
  const float om_dobj = dt > 0.0f ? std::fabs(s->rot_rad) / dt : 0.0f;
  const float om_wobj = dt > 0.0f ? std::fabs(s->wrot_rad) / dt : 0.0f;
  const float R = s->hp.drum_r;
  float v = 0.0f;
  if (s->cyl_rot) v = std::max(v, om_drum * R);
  for (int k = 0; k < s->n_d; ++k) {
    const DOBJ& D = s->d[k];
    for (int q = 0; q < D.num_vertex && q < 8; ++q) {
      if (s->hp.is_mill && D.is_attached_DWorld) v = std::max(v, om_drum * rxy(D.vertex[q], R, R));
      if (s->dobj_rot && D.is_attached_DWorld)
        v = std::max(v, om_dobj * rxy(D.vertex[q], s->rot_ax, s->rot_ay));
    }
    if (k == s->dobj_tr)
      v = std::max(v, std::sqrt(D.velocity.x * D.velocity.x + D.velocity.y * D.velocity.y +
                                D.velocity.z * D.velocity.z));
  }
  for (int k = 0; k < s->n_w; ++k) {
    const WOBJ& W = s->w[k];
    const bool turned = s->wobj_rot && k < 32 && ((s->wrot_mask >> k) & 1u);
    const bool drum_faces = s->hp.rotating_wobj && s->cyl_rot;
    for (int q = 0; q < W.num_vertex && q < 16; ++q) {
      if (turned) v = std::max(v, om_wobj * rxy(W.vertex[q], s->wrot_ax, s->wrot_ay));
      if (drum_faces) v = std::max(v, om_drum * rxy(W.vertex[q], R, R));
    }
  }
  return v;
}

// After a forced re-sort (new state, fill wave, removal, new options) the
// next regular check may be up to kListCheckEvery steps away and nothing has
// looked ahead from the new state: every step up to the next multiple of
// kListCheckEvery ends with a check, and those steps run as plain steps in
// both stepping modes, so graph and plain stepping re-sort at the same steps.
void force_check(blaze_sim* s) {
  s->check_until = (s->steps / kListCheckEvery + 1) * kListCheckEvery;
}

// Fill_State and the wave control of Device_DEM_UpdateSim
// (DeviceInterface.cu:1055-1110, 1840-1866): before a step, either the next
// wave joins (the counter passed the clearing time, or nothing is in the
// run yet) or the counter advances.  A wave is the next fill_pack particles
// at the end of the run, in memory order.
int fill_wave(blaze_sim* s) {
  if (s->fill_counter > s->fill_clear || s->fill_n == 0) {
    s->fill_counter = 0;
    if (s->fill_n < s->n_max) {
      s->fill_n += std::min(s->fill_pack, s->n_max - s->fill_n);
      CK(cudaStreamSynchronize(s->stream));
      CK(cudaMemcpy(&s->h_ctl->n_cur, &s->ctl->n_cur, sizeof(int), cudaMemcpyDeviceToHost));
      s->h_ctl->n_cur = s->fill_n;
      s->h_ctl->rebuild_req = 1;
      force_check(s);
      CK(cudaMemcpy(&s->ctl->n_cur, &s->h_ctl->n_cur, sizeof(int), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(&s->ctl->rebuild_req, &s->h_ctl->rebuild_req, sizeof(int),
                    cudaMemcpyHostToDevice));
    }
    if (s->fill_n >= s->n_max) s->filling = false;
  } else {
    s->fill_counter++;
  }
  return 0;
}

// Whether the step about to run starts a block of list checks, and whether
// it ends with a recorded check (list_needs_rebuild).
int block_start_here(const blaze_sim* s) {
  return (int)(s->opt.skin > 0.0f && s->steps % kListCheckEvery == 0 &&
               s->steps >= s->check_until);
}
int check_after_here(const blaze_sim* s) {
  return (int)((s->steps + 1) % kListCheckEvery == 0 || s->steps < s->check_until);
}

// After the kernels of one step: the next state is current; the removal
// check of a silo or plant every 1000 steps (DeviceInterface.cu:2463-2498).
void finish_step(blaze_sim* s) {
  s->cur ^= 1;
  s->steps++;
  if (s->si.Kill_Particles) {
    s->stepc++;
    if (s->stepc >= 1000) {
      launch_kill(s->S[s->cur], s->ob, s->n_max, s->si.Silo_Kill_Height,
                  s->si.Rotating_WObject ? 1 : 0, s->si.max_size, s->ctl, s->stream);
      force_check(s);
      s->last_launches += 1;
      s->stepc = 0;
    }
  }
}

int enqueue_step(blaze_sim* s) {
  if (s->filling) {
    int rc = fill_wave(s);
    if (rc) return rc;
  }
  if (s->profile) prof_event(s, 0);
  launch_gate(s->ctl, s->stream, s->opt.skin, list_look(s), block_start_here(s), wall_speed(s));
  int rc = enqueue_rebuild(s, &s->ctl->rebuilt, s->stream);
  if (rc) return rc;
  if (s->profile) { prof_event(s, 0); prof_event(s, 1); }
  s->last_launches += 1 + enqueue_step_kernels(
                              s, StepLink{&s->ctl->rebuilt, 0, 0, check_after_here(s)}, s->stream);
  if (s->profile) prof_event(s, 1);
  finish_step(s);
  return 0;
}

void drop_graphs(blaze_sim* s) {
  for (int c = 0; c < 2; ++c) {
    if (s->graph[c]) cudaGraphExecDestroy(s->graph[c]);
    s->graph[c] = nullptr;
    if (s->block[c]) cudaGraphExecDestroy(s->block[c]);
    s->block[c] = nullptr;
    for (int b = 0; b < 2; ++b)
      for (int k = 0; k < 2; ++k) {
        if (s->single[c][b][k]) cudaGraphExecDestroy(s->single[c][b][k]);
        s->single[c][b][k] = nullptr;
      }
  }
}

// Adds to the graph being captured on `cs` a conditional node of `type`
// with `nbody` bodies (IF: 1, or 2 for IF/ELSE; SWITCH: any) on handle h;
// returns the bodies.
int add_conditional(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    int nbody, cudaGraph_t* bodies) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t capg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  CK(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &capg, &deps, &ndeps));
  alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];
  std::memset(cp_raw, 0, sizeof(cp_raw));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = type;
  cp.conditional.size = (unsigned)nbody;
  cudaGraphNode_t cnode;
  CK(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
  for (int b = 0; b < nbody; ++b) bodies[b] = cp.conditional.phGraph_out[b];
  CK(cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies));
  return 0;
}

// An IF node on h (captured on `cs`) whose body, captured on `bs`, marks
// step k in d_rb (k >= 0), then re-sorts and rebuilds the neighbour list.
int add_rebuild_if(blaze_sim* s, cudaStream_t cs, cudaStream_t bs, cudaGraphConditionalHandle h,
                   int k) {
  cudaGraph_t body = nullptr;
  int rc = add_conditional(cs, h, cudaGraphCondTypeIf, 1, &body);
  if (rc) return rc;
  CK(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  if (k >= 0) CK(cudaMemsetAsync(s->d_rb + k, 0x01, sizeof(int), bs));
  rc = enqueue_rebuild(s, nullptr, bs);
  cudaGraph_t tmp = nullptr;
  CK(cudaStreamEndCapture(bs, &tmp));
  return rc;
}

// kGraphSteps steps as one CUDA graph, starting from S[c], without a skin
// (the reference re-sorts every step): a one-thread gate kernel carries the
// re-sort request of the previous launch into the first step's IF node, and
// every later step's IF condition is set by the step kernel before it.  An
// IF body marks its step in d_rb, then re-sorts and rebuilds the neighbour
// list.  Steps that keep the list launch only the fused step kernel.
int build_graph(blaze_sim* s, int c) {
  const int saved = s->cur;
  s->cur = c;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h[kGraphSteps];
  for (int k = 0; k < kGraphSteps; ++k)
    CK(cudaGraphConditionalHandleCreate(&h[k], g, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(s->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  launch_gate_graph(s->ctl, h[0], s->d_rb, kGraphSteps, s->stream);
  int rc = 0;
  for (int k = 0; k < kGraphSteps && !rc; ++k) {
    rc = add_rebuild_if(s, s->stream, s->aux, h[k], k);
    const StepLink link = k + 1 < kGraphSteps ? StepLink{s->d_rb + k, h[k + 1], 1, 1}
                                               : StepLink{s->d_rb + k, 0, 0, 1};
    s->step_launches = enqueue_step_kernels(s, link, s->stream);
    s->cur ^= 1;
  }
  cudaGraph_t out = nullptr;
  CK(cudaStreamEndCapture(s->stream, &out));
  if (!rc) CK(cudaGraphInstantiate(&s->graph[c], out, 0));
  CK(cudaGraphDestroy(out));
  s->cur = saved;
  return rc;
}

// With a skin, graph stepping runs blocks of kListCheckEvery steps
// (list_needs_rebuild).  A block is one graph: the block-start gate, then a
// SWITCH node whose body the gate picks on the device, so no block waits
// for the host:
//   0 keep   the kGraphSteps step kernels;
//   1 re-sort, then the step kernels (the first reads the sorted copy);
//   2 exact  an IF node (re-sort) before every step, set by the step before.
enum BlockKind { kBlockKeep = 0, kBlockResort = 1, kBlockExact = 2 };

// Captures into `body` (on stream bs; nested IF bodies on bs2) the steps of
// one block kind starting from S[c].
int capture_block_body(blaze_sim* s, cudaGraph_t body, cudaStream_t bs, cudaStream_t bs2, int c,
                       int kind) {
  s->cur = c;
  const int n_if = kind == kBlockExact ? kGraphSteps : 0;
  cudaGraphConditionalHandle h[kGraphSteps];
  for (int k = 0; k < n_if; ++k)
    CK(cudaGraphConditionalHandleCreate(&h[k], body, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  if (kind == kBlockResort) rc = enqueue_rebuild(s, nullptr, bs);
  if (kind == kBlockExact) launch_gate_body(s->ctl, h[0], bs);
  for (int k = 0; k < kGraphSteps && !rc; ++k) {
    if (k < n_if) rc = add_rebuild_if(s, bs, bs2, h[k], k);
    const StepLink link = k + 1 < n_if ? StepLink{s->d_rb + k, h[k + 1], 1, 0}
                                        : StepLink{s->d_rb + k, 0, 0, (int)(k + 1 == kGraphSteps)};
    s->step_launches = enqueue_step_kernels(s, link, bs);
    s->cur ^= 1;
  }
  cudaGraph_t tmp = nullptr;
  CK(cudaStreamEndCapture(bs, &tmp));
  return rc;
}

int build_block(blaze_sim* s, int c) {
  const int saved = s->cur;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hs;
  CK(cudaGraphConditionalHandleCreate(&hs, g, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(s->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  launch_gate_switch(s->ctl, hs, s->d_rb, kGraphSteps, s->opt.skin, list_look(s), wall_speed(s),
                     s->stream);
  cudaGraph_t bodies[3] = {nullptr, nullptr, nullptr};
  int rc = add_conditional(s->stream, hs, cudaGraphCondTypeSwitch, 3, bodies);
  for (int kind = 0; kind < 3 && !rc; ++kind)
    rc = capture_block_body(s, bodies[kind], s->aux, s->aux2, c, kind);
  cudaGraph_t out = nullptr;
  CK(cudaStreamEndCapture(s->stream, &out));
  if (!rc) CK(cudaGraphInstantiate(&s->block[c], out, 0));
  CK(cudaGraphDestroy(out));
  s->cur = saved;
  return rc;
}

// One step with a skin as a graph, starting from S[c]: the gate of plain
// stepping (block start or not), an IF node re-sorting when it says so, and
// the step kernels (recording a list check after the step or not).  Steps
// outside whole blocks (a tail shorter than a block, the steps after a
// forced re-sort, those around a removal check) run this way; they make the
// decisions plain stepping makes, with an IF node instead of gated kernels.
int build_single(blaze_sim* s, int c, int bstart, int chk) {
  const int saved = s->cur;
  s->cur = c;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(s->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  launch_gate_if(s->ctl, h, s->opt.skin, list_look(s), bstart, wall_speed(s), s->stream);
  int rc = add_rebuild_if(s, s->stream, s->aux, h, -1);
  if (!rc) s->step_launches = enqueue_step_kernels(s, StepLink{&s->ctl->rebuilt, 0, 0, chk},
                                                   s->stream);
  cudaGraph_t out = nullptr;
  CK(cudaStreamEndCapture(s->stream, &out));
  if (!rc) CK(cudaGraphInstantiate(&s->single[c][bstart][chk], out, 0));
  CK(cudaGraphDestroy(out));
  s->cur = saved;
  return rc;
}

// Instantiates every graph the current options can launch, so that no
// stream capture or instantiation happens inside a later blaze_step.
int prepare_graphs(blaze_sim* s) {
  for (int c = 0; c < 2; ++c) {
    if (s->opt.skin > 0.0f) {
      if (!s->block[c]) {
        int rc = build_block(s, c);
        if (rc) return rc;
      }
      for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 2; ++k)
          if (!s->single[c][b][k]) {
            int rc = build_single(s, c, b, k);
            if (rc) return rc;
          }
    } else if (!s->graph[c]) {
      int rc = build_graph(s, c);
      if (rc) return rc;
    }
  }
  return 0;
}

int graph_steps(blaze_sim* s, int nsteps) {
  int rc = prepare_graphs(s);
  if (rc) return rc;
  int done = 0;
  while (done < nsteps) {
    // a removal check every 1000 steps ends a step outside a block
    const bool kill_soon = s->si.Kill_Particles && s->stepc + kGraphSteps >= 1000;
    const int c = s->cur;
    if (s->opt.skin > 0.0f) {
      if (nsteps - done >= kGraphSteps && !kill_soon && block_start_here(s)) {
        CK(cudaGraphLaunch(s->block[c], s->stream));
        // the gate and the step kernels (re-sorts and the exact mode's
        // extra gate are counted on the device)
        s->last_launches += 1 + kGraphSteps * s->step_launches;
        s->steps += kGraphSteps;
        if (s->si.Kill_Particles) s->stepc += kGraphSteps;
        if (kGraphSteps & 1) s->cur ^= 1;
        done += kGraphSteps;
      } else {
        CK(cudaGraphLaunch(s->single[c][block_start_here(s)][check_after_here(s)], s->stream));
        s->last_launches += 1 + s->step_launches;
        finish_step(s);
        done += 1;
      }
      continue;
    }
    if (nsteps - done < kGraphSteps || kill_soon) {
      rc = enqueue_step(s);
      if (rc) return rc;
      done += 1;
      continue;
    }
    CK(cudaGraphLaunch(s->graph[c], s->stream));
    // launches that always run: the gate and the step kernels of each step
    // (re-sort bodies run only when a step asks for them)
    s->last_launches += 1 + kGraphSteps * s->step_launches;
    s->steps += kGraphSteps;
    if (s->si.Kill_Particles) s->stepc += kGraphSteps;
    if (kGraphSteps & 1) s->cur ^= 1;
    done += kGraphSteps;
  }
  return 0;
}

int sync_status(blaze_sim* s) {
  CK(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  s->status |= s->h_ctl->status;
  return (int)s->status;
}

int set_state_impl(blaze_sim* s, const float* pos3, const float* quat4, const float* vel3,
                   const float* avel3, const uint* type, const int* pid) {
  const int n = s->n_max;
  int rc = sync_status(s);
  if (rc < 0) return rc;
  const int e = s->h_ctl->epoch & 1;
  const HostStage& hs = s->stage;
  CK(cudaMemsetAsync(hs.flags, 0, 2 * sizeof(int), s->stream));
  CK(cudaMemcpyAsync(hs.pos3, pos3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->stream));
  if (vel3)
    CK(cudaMemcpyAsync(hs.vel3, vel3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->stream));
  if (avel3)
    CK(cudaMemcpyAsync(hs.avel3, avel3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(hs.type, type, sizeof(uint) * n, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(hs.pid, pid, sizeof(int) * n, cudaMemcpyHostToDevice, s->stream));
  const bool has_q = s->poly && quat4 != nullptr;
  if (has_q)
    CK(cudaMemcpyAsync(hs.quat4, quat4, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, s->stream));
  launch_pack_state(s->dp, hs, vel3 != nullptr, avel3 != nullptr, s->S[s->cur], s->ob.pid[e],
                    s->n_d > 0 ? s->ob.lift[e] : nullptr, s->poly ? s->ob.ornt[e] : nullptr,
                    has_q, n, s->stream);
  CK(cudaMemcpyAsync(s->h_flags, hs.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  const int dead = s->h_flags[0];
  const bool spin_free = !s->poly && !s->si.Rotation && s->h_flags[1] == 0;
  if (spin_free != s->spin_free) {
    drop_graphs(s);
    s->spin_free = spin_free;
  }
  StepCtl c = *s->h_ctl;
  c.rebuild_req = 1;
  c.rebuilt = 0;
  c.n_cur = n;
  c.pending_dead = dead;
  *s->h_ctl = c;
  CK(cudaMemsetAsync(s->d_chk, 0, sizeof(uint32_t) * 2 * kChkSlots * kChkStride, s->stream));
  force_check(s);
  CK(cudaMemcpyAsync(s->ctl, s->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int get_state_impl(blaze_sim* s, float* pos3, float* quat4, float* vel3, float* avel3, uint* type,
                   int* pid) {
  int st = sync_status(s);
  if (st < 0) return st;
  const int n = s->n_max;
  const int e = s->h_ctl->epoch & 1;
  const HostStage& hs = s->stage;
  launch_unpack_state(s->dp, hs, s->S[s->cur], s->ob.pid[e], s->poly ? s->ob.ornt[e] : nullptr, n,
                      s->stream);
  if (quat4 && s->poly)
    CK(cudaMemcpyAsync(quat4, hs.quat4, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost, s->stream));
  if (pos3) CK(cudaMemcpyAsync(pos3, hs.pos3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
  if (vel3) CK(cudaMemcpyAsync(vel3, hs.vel3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
  if (avel3) CK(cudaMemcpyAsync(avel3, hs.avel3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s->stream));
  if (type) CK(cudaMemcpyAsync(type, hs.type, sizeof(uint) * n, cudaMemcpyDeviceToHost, s->stream));
  if (pid) CK(cudaMemcpyAsync(pid, hs.pid, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  return st;
}

void free_sim(blaze_sim* s) {
  if (!s) return;
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (int b = 0; b < 3; ++b) { f(s->S[b].pos); f(s->S[b].vel); f(s->S[b].angv); }
  for (int b = 0; b < 2; ++b) { f(s->ob.pid[b]); f(s->ob.lift[b]); f(s->rs.keys[b]); f(s->rs.vals[b]); }
  f(s->rs.counts); f(s->rs.totals); f(s->cstart); f(s->cend); f(s->nl.idx); f(s->nl.cnt);
  f(s->ctl); f(s->d_rb); f(s->d_chk); f(s->dp); f(s->d_ops); f(s->d_wall_off); f(s->d_wall_idx);
  f(s->d_tally); f(s->d_eb); f(s->d_epart);
  f(s->cap.f_pp); f(s->cap.t_pp); f(s->cap.f_w); f(s->cap.t_w); f(s->cap.f_l); f(s->cap.t_l);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  f(s->stage.pos3); f(s->stage.vel3); f(s->stage.avel3); f(s->stage.type); f(s->stage.pid);
  f(s->stage.flags); f(s->stage.quat4);
  f(s->ob.ornt[0]); f(s->ob.ornt[1]); f(s->d_shapes);
  f(s->geom.vert); f(s->geom.fnorm); f(s->geom.fcent);
  f(s->pairs.status); f(s->pairs.hint); f(s->pairs.con); f(s->pairs.qv); f(s->pairs.qe); f(s->pairs.counts);
  f(s->nl.flat);
  f(s->d_count);
  if (s->h_flags) cudaFreeHost(s->h_flags);
  for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
  drop_graphs(s);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->aux) cudaStreamDestroy(s->aux);
  if (s->aux2) cudaStreamDestroy(s->aux2);
  delete s;
}

// A polyhedral particle object must fit the fixed-size tables of POBJ and
// index only its own vertices.
bool poly_object_valid(const POBJ& o, int t) {
  auto bad = [&](const char* what) {
    std::fprintf(stderr, "blaze: polyhedral particle object %d: %s\n", t, what);
    return false;
  };
  if (o.num_vertex < 1 || o.num_vertex > kPolyMaxV) return bad("num_vertex outside 1..32");
  if (o.num_faces < 1 || o.num_faces > kPolyMaxF) return bad("num_faces outside 1..32");
  if (o.num_edges < 0 || o.num_edges > kPolyMaxE) return bad("num_edges outside 0..32");
  for (int f = 0; f < o.num_faces; ++f) {
    const Surface& F = o.face[f];
    if (F.num_vertex < 1 || F.num_vertex > kPolyFaceV) return bad("face vertex count outside 1..8");
    for (int k = 0; k < F.num_vertex; ++k)
      if (F.vertex_Order[k] < 0 || F.vertex_Order[k] >= o.num_vertex)
        return bad("face vertex index outside the object");
  }
  for (int e = 0; e < o.num_edges; ++e)
    for (int k = 0; k < 2; ++k)
      if (o.edge[e].point_vindex[k] >= (uint)o.num_vertex)
        return bad("edge vertex index outside the object");
  return true;
}

// Body-frame objects to the device, orientation copies, world-frame
// geometry buffers sized by the largest object, orientation staging.
int setup_poly(blaze_sim* s) {
  std::vector<PolyShape> shapes(kMaxTypes);
  std::memset(shapes.data(), 0, sizeof(PolyShape) * kMaxTypes);
  int kv = 1, kf = 1;
  for (int t = 0; t < s->n_p; ++t) {
    const POBJ& o = s->p[t];
    PolyShape& S = shapes[t];
    S.nv = o.num_vertex;
    S.nf = o.num_faces;
    S.ne = o.num_edges;
    for (int k = 0; k < S.nv; ++k)
      S.vert[k] = make_float4(o.Local_Vertex[k].x, o.Local_Vertex[k].y, o.Local_Vertex[k].z, 0.0f);
    for (int f = 0; f < S.nf; ++f) {
      const Surface& F = o.face[f];
      S.fnorm[f] = make_float4(F.normal.x, F.normal.y, F.normal.z, 0.0f);
      // face.centroid - COM, the body-frame offset RotatePolyhedra rotates
      S.fcent[f] = make_float4(F.centroid.x - o.COM.x, F.centroid.y - o.COM.y,
                               F.centroid.z - o.COM.z, 0.0f);
      S.farea[f] = F.area;
      S.fnv[f] = F.num_vertex;
      for (int k = 0; k < F.num_vertex; ++k) S.ford[f][k] = (uint8_t)F.vertex_Order[k];
    }
    for (int e = 0; e < S.ne; ++e) {
      S.edge[e][0] = (uint8_t)o.edge[e].point_vindex[0];
      S.edge[e][1] = (uint8_t)o.edge[e].point_vindex[1];
    }
    for (int k = 0; k < 9; ++k) S.inertia[k] = o.InertiaT[k];
    S.com[0] = o.COM.x; S.com[1] = o.COM.y; S.com[2] = o.COM.z;
    // bounds the edge-edge pruning relies on, rounded up (rotation preserves
    // lengths up to a few units in the last place)
    double rmax = 0.0, emax = 0.0;
    for (int k = 0; k < S.nv; ++k) {
      const double x = o.Local_Vertex[k].x, y = o.Local_Vertex[k].y, z = o.Local_Vertex[k].z;
      rmax = std::max(rmax, std::sqrt(x * x + y * y + z * z));
    }
    for (int e = 0; e < S.ne; ++e) {
      const float3 a = o.Local_Vertex[S.edge[e][0]], b = o.Local_Vertex[S.edge[e][1]];
      const double dx = (double)b.x - a.x, dy = (double)b.y - a.y, dz = (double)b.z - a.z;
      emax = std::max(emax, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    S.rmax = (float)(rmax * (1.0 + 1e-5) + 1e-6);
    S.emax = (float)(emax * (1.0 + 1e-5) + 1e-6);
    kv = std::max(kv, S.nv);
    kf = std::max(kf, S.nf);
  }
  const size_t n = (size_t)s->n_max;
  CK(dalloc(&s->d_shapes, kMaxTypes));
  CK(cudaMemcpy(s->d_shapes, shapes.data(), sizeof(PolyShape) * kMaxTypes,
                cudaMemcpyHostToDevice));
  s->geom.kv = kv;
  s->geom.kf = kf;
  CK(dalloc(&s->geom.vert, n * kv));
  CK(dalloc(&s->geom.fnorm, n * kf));
  CK(dalloc(&s->geom.fcent, n * kf));
  for (int b = 0; b < 2; ++b) {
    CK(dalloc(&s->ob.ornt[b], n));
    std::vector<float4> ident(n, make_float4(1.0f, 0.0f, 0.0f, 0.0f));
    CK(cudaMemcpy(s->ob.ornt[b], ident.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
  }
  CK(dalloc(&s->stage.quat4, 4 * n));
  s->poly = true;
  return alloc_poly_pairs(s);
}

int create_impl(blaze_sim** out, const WOBJ* w, int n_w, const POBJ* p, int n_p, const DOBJ* d,
                int n_d, const SimulationInfo* si, const blaze_options* opt) {
  if (!out || !si || n_w < 0 || n_w > 8 || n_p < 1 || n_p > kMaxTypes || n_d < 0 ||
      n_d > kMaxDobj || si->Num_Particles <= 0 || (n_w && !w) || !p || (n_d && !d))
    return -1;
  if (si->particle_type != 0 && si->particle_type != 1) {
    std::fprintf(stderr, "blaze: particle_type %d is not supported (0 spheres, 1 polyhedra)\n",
                 si->particle_type);
    return -1;
  }
  if (si->particle_type == 1) {
    for (int t = 0; t < n_p; ++t)
      if (!poly_object_valid(p[t], t)) return -1;
  }
  blaze_sim* s = new (std::nothrow) blaze_sim();
  if (!s) return -1;
  s->n_max = si->Num_Particles;
  s->si = *si;
  s->si.Num_ParticlesPerObject = nullptr;
  if (n_w) std::memcpy(s->w, w, sizeof(WOBJ) * n_w);
  std::memcpy(s->p, p, sizeof(POBJ) * n_p);
  if (n_d) std::memcpy(s->d, d, sizeof(DOBJ) * n_d);
  s->n_w = n_w; s->n_p = n_p; s->n_d = n_d;
  s->num_wobj = si->Num_WorldObjects;
  if (opt) s->opt = *opt;
  else blaze_default_options(&s->opt);
  if (s->opt.max_nbr <= 0) s->opt.max_nbr = 32;
  if (s->opt.max_nbr > 32) {  // the reference's 32 slots; the step masks them in 32 bits
    std::fprintf(stderr, "blaze: max_nbr %d exceeds 32 neighbour slots\n", s->opt.max_nbr);
    delete s;
    return -1;
  }
  const int n = s->n_max;
  auto fail = [&](int rc) { free_sim(s); return rc; };
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  e = cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  e = cudaStreamCreateWithFlags(&s->aux2, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(cuda_fail(e));
#define CKF(x) do { cudaError_t e2 = (x); if (e2 != cudaSuccess) return fail(cuda_fail(e2)); } while (0)
  for (int b = 0; b < 3; ++b) {
    CKF(dalloc(&s->S[b].pos, n)); CKF(dalloc(&s->S[b].vel, n)); CKF(dalloc(&s->S[b].angv, n));
  }
  for (int b = 0; b < 2; ++b) {
    CKF(dalloc(&s->ob.pid[b], n));
    CKF(dalloc(&s->ob.lift[b], n));
    CKF(dalloc(&s->rs.keys[b], n));
    CKF(dalloc(&s->rs.vals[b], n));
  }
  const int tiles = (n + kTileKeys - 1) / kTileKeys;
  s->rs.max_n = n;
  s->rs.max_tiles = tiles;
  CKF(dalloc(&s->rs.counts, (size_t)kRadixDigits * std::max(tiles, 1)));
  CKF(dalloc(&s->rs.totals, kRadixDigits));
  CKF(dalloc(&s->dp, 1));
  CKF(dalloc(&s->ctl, 1));
  CKF(dalloc(&s->d_rb, kGraphSteps));
  CKF(cudaMemset(s->d_rb, 0, sizeof(int) * kGraphSteps));
  CKF(dalloc(&s->d_tally, 3));
  CKF(cudaMemset(s->d_tally, 0, sizeof(double) * 3));
  if (si->EnergyCalc) {
    CKF(dalloc(&s->d_eb, (size_t)3 * n));
    CKF(dalloc(&s->d_epart, (size_t)3 * ((n + kEnergyBlock - 1) / kEnergyBlock)));
  }
  CKF(cudaMallocHost((void**)&s->h_ctl, sizeof(StepCtl)));
  CKF(dalloc(&s->stage.pos3, (size_t)3 * n));
  CKF(dalloc(&s->stage.vel3, (size_t)3 * n));
  CKF(dalloc(&s->stage.avel3, (size_t)3 * n));
  CKF(dalloc(&s->stage.type, n));
  CKF(dalloc(&s->stage.pid, n));
  CKF(dalloc(&s->stage.flags, 2));
  CKF(cudaMallocHost((void**)&s->h_flags, 2 * sizeof(int)));
  CKF(dalloc(&s->d_count, 1));
  std::memset(s->h_ctl, 0, sizeof(StepCtl));
  CKF(dalloc(&s->d_chk, (size_t)2 * kChkSlots * kChkStride));
  CKF(cudaMemset(s->d_chk, 0, sizeof(uint32_t) * 2 * kChkSlots * kChkStride));
  s->h_ctl->chk = s->d_chk;
  s->h_ctl->n_cur = n;
  s->h_ctl->rebuild_req = 1;
  force_check(s);
  CKF(cudaMemcpy(s->ctl, s->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice));
  int rc = upload_params(s);
  if (rc) return fail(rc);
  rc = alloc_cells(s);
  if (rc) return fail(rc);
  rc = alloc_nlist(s);
  if (rc) return fail(rc);
  rc = alloc_capture(s);
  if (rc) return fail(rc);
  if (si->particle_type == 1) {
    rc = setup_poly(s);
    if (rc) return fail(rc);
  }
  // zero state until the caller sets one (Set_Init_Config_Device zeroes velocities)
  for (int b = 0; b < 3; ++b) {
    CKF(cudaMemset(s->S[b].pos, 0, sizeof(float4) * n));
    CKF(cudaMemset(s->S[b].vel, 0, sizeof(float4) * n));
    CKF(cudaMemset(s->S[b].angv, 0, sizeof(float4) * n));
  }
  for (int b = 0; b < 2; ++b) {
    CKF(cudaMemset(s->ob.pid[b], 0, sizeof(int) * n));
    CKF(cudaMemset(s->ob.lift[b], 0xff, sizeof(int) * n));
  }
  CKF(cudaDeviceSynchronize());
#undef CKF
  *out = s;
  return 0;
}

}  // namespace

// ======================================================================= ABI
extern "C" {

void blaze_default_options(blaze_options* o) {
  if (!o) return;
  o->skin = 0.0f;
  o->max_nbr = 32;
  o->wall_grid = 1;
  o->use_graph = 0;
  o->capture_forces = 0;
  o->sync_each_step = 0;
  o->fast_law = 0;
}

int blaze_create(blaze_sim** out, const WOBJ* w, int n_w, const POBJ* p, int n_p, const DOBJ* d,
                 int n_d, const SimulationInfo* si, const blaze_options* opt) {
  return create_impl(out, w, n_w, p, n_p, d, n_d, si, opt);
}

int blaze_destroy(blaze_sim* s) {
  if (!s) return -1;
  if (s == g_default) g_default = nullptr;
  cudaStreamSynchronize(s->stream);
  free_sim(s);
  return 0;
}

int blaze_set_options(blaze_sim* s, const blaze_options* opt) {
  if (!s || !opt) return -1;
  const blaze_options old = s->opt;
  if (opt->max_nbr > 32) {  // the reference's 32 slots; the step masks them in 32 bits
    std::fprintf(stderr, "blaze: max_nbr %d exceeds 32 neighbour slots\n", opt->max_nbr);
    return -1;
  }
  s->opt = *opt;
  if (s->opt.max_nbr <= 0) s->opt.max_nbr = 32;
  CK(cudaStreamSynchronize(s->stream));
  int rc = 0;
  if (s->opt.max_nbr != old.max_nbr) rc = alloc_nlist(s);
  if (!rc) rc = alloc_capture(s);
  if (!rc) rc = upload_params(s);
  // a skin turned on or off changes the list grid
  if (!rc) rc = alloc_cells(s);
  // a new skin or capacity invalidates the current list
  s->h_ctl->rebuild_req = 1;
  force_check(s);
  CK(cudaMemcpy(&s->ctl->rebuild_req, &s->h_ctl->rebuild_req, sizeof(int), cudaMemcpyHostToDevice));
  return rc;
}

int blaze_set_cylinder_rotation(blaze_sim* s, int on) {
  if (!s) return -1;
  int rc = pull_dobj(s);
  if (rc) return rc;
  s->cyl_rot = on ? 1 : 0;
  s->hp.cyl_rot = s->cyl_rot;
  drop_graphs(s);   // the list check's wall speed changes
  CK(cudaMemcpyAsync(s->dp, &s->hp, sizeof(SimParams), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int blaze_set_state(blaze_sim* s, const float* pos3, const float* vel3, const float* avel3,
                    const uint* type, const int* pid) {
  if (!s || !pos3 || !type || !pid) return -1;
  return set_state_impl(s, pos3, nullptr, vel3, avel3, type, pid);
}

int blaze_get_state(blaze_sim* s, float* pos3, float* vel3, float* avel3, uint* type, int* pid) {
  if (!s) return -1;
  return get_state_impl(s, pos3, nullptr, vel3, avel3, type, pid);
}

int blaze_set_state_ornt(blaze_sim* s, const float* pos3, const float* quat4, const float* vel3,
                         const float* avel3, const uint* type, const int* pid) {
  if (!s || !pos3 || !type || !pid) return -1;
  return set_state_impl(s, pos3, quat4, vel3, avel3, type, pid);
}

int blaze_get_state_ornt(blaze_sim* s, float* pos3, float* quat4, float* vel3, float* avel3,
                         uint* type, int* pid) {
  if (!s) return -1;
  return get_state_impl(s, pos3, quat4, vel3, avel3, type, pid);
}

int blaze_step(blaze_sim* s, int nsteps) {
  if (!s || nsteps < 0) return -1;
  s->last_launches = 0;
  if (s->opt.use_graph && !s->opt.sync_each_step && !s->profile && !s->filling) {
    int rc = graph_steps(s, nsteps);
    if (rc) return rc;
    CK(cudaGetLastError());
    return 0;
  }
  for (int k = 0; k < nsteps; ++k) {
    int rc = enqueue_step(s);
    if (rc) return rc;
    if (s->opt.sync_each_step) {
      rc = sync_status(s);
      if (rc != 0) return rc;
    }
  }
  CK(cudaGetLastError());
  return s->opt.sync_each_step ? (int)s->status : 0;
}

int blaze_sync(blaze_sim* s) {
  if (!s) return -1;
  return sync_status(s);
}

int blaze_prepare_graphs(blaze_sim* s) {
  if (!s) return -1;
  int rc = prepare_graphs(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int blaze_num_exact_blocks(blaze_sim* s) {
  if (!s) return -1;
  int rc = sync_status(s);
  if (rc < 0) return rc;
  return s->h_ctl->exact_blocks;
}

int blaze_num_current(blaze_sim* s) {
  if (!s) return -1;
  int rc = sync_status(s);
  if (rc < 0) return rc;
  return s->h_ctl->n_cur - s->h_ctl->pending_dead;
}

int blaze_num_rebuilds(blaze_sim* s) {
  if (!s) return -1;
  int rc = sync_status(s);
  if (rc < 0) return rc;
  return s->h_ctl->epoch;
}

int blaze_update_wobj(blaze_sim* s, const WOBJ* w, int n_w) {
  if (!s || !w || n_w < 0 || n_w > 8) return -1;
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(s->w, w, sizeof(WOBJ) * n_w);
  s->wobj_on_device = false;   // the caller's objects replace the turned ones
  // moving geometry: the per-cell culling lists would go stale
  s->walls_static = false;
  return upload_params(s);
}

int blaze_update_dobj(blaze_sim* s, const DOBJ* d, int n_d) {
  if (!s || !d || n_d < 0 || n_d > kMaxDobj) return -1;
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(s->d, d, sizeof(DOBJ) * n_d);
  s->dobj_on_device = false;   // the caller's objects replace the turned ones
  build_params(s);
  CK(cudaMemcpyAsync(s->dp, &s->hp, sizeof(SimParams), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int blaze_set_dobj_rotation(blaze_sim* s, float about_x, float about_y, float rad_per_step,
                            int on) {
  if (!s) return -1;
  CK(cudaStreamSynchronize(s->stream));
  s->dobj_rot = on != 0 && s->n_d > 0;
  if (s->dobj_rot) s->dobj_on_device = true;
  s->rot_ax = about_x;
  s->rot_ay = about_y;
  // the host's single-precision cosine and sine of the step angle, as the
  // drum driver evaluates them once per step (Processing_Mills.h:20-21)
  s->rot_c = std::cos(rad_per_step);
  s->rot_s = std::sin(rad_per_step);
  s->rot_rad = rad_per_step;
  drop_graphs(s);
  return 0;
}

int blaze_set_dobj_translation(blaze_sim* s, int index, int on) {
  if (!s || (on && (index < 0 || index >= s->n_d))) return -1;
  CK(cudaStreamSynchronize(s->stream));
  s->dobj_tr = on ? index : -1;
  if (on) s->dobj_on_device = true;
  drop_graphs(s);
  return 0;
}

int blaze_set_wobj_rotation(blaze_sim* s, float about_x, float about_y, float rad_per_step,
                            int on) {
  if (!s) return -1;
  int rc = pull_wobj(s);
  if (rc) return rc;
  s->wrot_mask = 0;
  for (int k = 0; k < s->n_w && k < 32; ++k)
    if (s->w[k].is_rotating) s->wrot_mask |= 1u << k;
  s->wobj_rot = on != 0 && s->wrot_mask != 0;
  s->wrot_ax = about_x;
  s->wrot_ay = about_y;
  s->wrot_c = std::cos(rad_per_step);   // the host's single-precision cosine and sine
  s->wrot_s = std::sin(rad_per_step);   // (Processing_Mills.h:269-270)
  s->wrot_rad = rad_per_step;
  // moving walls: no per-cell candidate lists
  if (s->wobj_rot) s->walls_static = false;
  rc = upload_walls(s);
  if (s->wobj_rot) s->wobj_on_device = true;
  return rc;
}

int blaze_get_wobj(blaze_sim* s, WOBJ* w, int n_w) {
  if (!s || !w || n_w < 0) return -1;
  int rc = pull_wobj(s);
  if (rc) return rc;
  std::memcpy(w, s->w, sizeof(WOBJ) * std::min(n_w, s->n_w));
  return 0;
}

int blaze_get_dobj(blaze_sim* s, DOBJ* d, int n_d) {
  if (!s || !d || n_d < 0) return -1;
  int rc = pull_dobj(s);
  if (rc) return rc;
  std::memcpy(d, s->d, sizeof(DOBJ) * std::min(n_d, s->n_d));
  return 0;
}

int blaze_get_energy(blaze_sim* s, double* e3) {
  if (!s || !e3) return -1;
  CK(cudaStreamSynchronize(s->stream));
  double t[3];
  CK(cudaMemcpy(t, s->d_tally, sizeof(t), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 3; ++k) e3[k] = t[k] * 1E-4;
  return 0;
}

int blaze_set_energy(blaze_sim* s, const double* raw3) {
  if (!s) return -1;
  CK(cudaStreamSynchronize(s->stream));
  double t[3] = {0.0, 0.0, 0.0};
  if (raw3) for (int k = 0; k < 3; ++k) t[k] = raw3[k];
  CK(cudaMemcpy(s->d_tally, t, sizeof(t), cudaMemcpyHostToDevice));
  return 0;
}

long long blaze_check_division(long long n, unsigned long long seed) {
  if (n < 0) return -1;
  unsigned long long* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(*d)) != cudaSuccess) return -1;
  unsigned long long h = 0;
  cudaMemset(d, 0, sizeof(*d));
  launch_check_div(n, seed, d, 0);
  const cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? (long long)h : -1;
}

int blaze_write_state(blaze_sim* s, const char* path, const blaze_state_header* h) {
  if (!s || !path || !h) return -1;
  const int n = s->n_max;
  std::vector<float> pos(3 * n), q(4 * n), vel(3 * n), avel(3 * n), acc(3 * n, 0.0f);
  std::vector<uint> type(n);
  std::vector<int> pid(n);
  int rc = get_state_impl(s, pos.data(), s->poly ? q.data() : nullptr, vel.data(), avel.data(),
                          type.data(), pid.data());
  if (rc < 0) return rc;
  // the removed particles sit after the ones in the run
  const int cur = s->h_ctl->n_cur - s->h_ctl->pending_dead;
  return blaze_write_state_arrays(path, h, cur, pos.data(), q.data(), vel.data(), avel.data(),
                                  acc.data(), type.data(), pid.data(), s->p, s->n_p);
}

int blaze_get_forces(blaze_sim* s, float* f_pp, float* t_pp, float* f_w, float* t_w, float* f_l,
                     float* t_l) {
  if (!s || !s->cap_alloc) return -1;
  int st = sync_status(s);
  if (st < 0) return st;
  float* dst[6] = {f_pp, t_pp, f_w, t_w, f_l, t_l};
  float* src[6] = {s->cap.f_pp, s->cap.t_pp, s->cap.f_w, s->cap.t_w, s->cap.f_l, s->cap.t_l};
  for (int q = 0; q < 6; ++q)
    if (dst[q]) CK(cudaMemcpy(dst[q], src[q], sizeof(float) * 3 * s->n_max, cudaMemcpyDeviceToHost));
  return st;
}

int blaze_get_nlist(blaze_sim* s, uint* nn, uint* list) {
  if (!s || !nn || !list) return -1;
  int st = sync_status(s);
  if (st < 0) return st;
  const int n = s->n_max, cap = s->nl.cap;
  std::vector<uint32_t> cnt(n), idx((size_t)n * cap);
  CK(cudaMemcpy(cnt.data(), s->nl.cnt, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(idx.data(), s->nl.idx, sizeof(uint32_t) * (size_t)n * cap, cudaMemcpyDeviceToHost));
  const int live = s->h_ctl->n_cur;
  for (int i = 0; i < n; ++i) {
    nn[i] = i < live ? cnt[i] : 0u;
    for (int k = 0; k < cap; ++k)
      list[(size_t)i * cap + k] = (i < live && k < (int)cnt[i]) ? idx[(size_t)k * n + i] : 0u;
  }
  return st;
}

int blaze_device_state(blaze_sim* s, void** pos4, void** vel4, void** angv4, void** stream) {
  if (!s) return -1;
  if (pos4) *pos4 = s->S[s->cur].pos;
  if (vel4) *vel4 = s->S[s->cur].vel;
  if (angv4) *angv4 = s->S[s->cur].angv;
  if (stream) *stream = (void*)s->stream;
  return 0;
}

int blaze_device_view(blaze_sim* s, const void** pos4, const void** ornt4, int* n, void** stream) {
  if (!s) return -1;
  const int rc = sync_status(s);
  if (rc < 0) return rc;
  if (pos4) *pos4 = s->S[s->cur].pos;
  // orientations follow the particles' memory order, which changes at a
  // re-sort: the copy the step wrote is selected by the re-sort count
  if (ornt4) *ornt4 = s->poly ? s->ob.ornt[s->h_ctl->epoch & 1] : nullptr;
  if (n) *n = s->h_ctl->n_cur;
  if (stream) *stream = (void*)s->stream;
  return rc;
}

int blaze_count_above(blaze_sim* s, float height, int* count) {
  if (!s || !count) return -1;
  CK(cudaMemsetAsync(s->d_count, 0, sizeof(unsigned int), s->stream));
  launch_count_above(s->S[s->cur].pos, s->ctl, s->n_max, height, s->d_count, s->stream);
  CK(cudaMemcpyAsync(s->h_flags, s->d_count, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                     s->stream));
  const int rc = sync_status(s);
  *count = s->h_flags[0];
  return rc;
}

int blaze_last_launches(blaze_sim* s) { return s ? s->last_launches : -1; }

int blaze_rebuild_kernels(blaze_sim* s) {
  if (!s) return -1;
  return 3 + 3 * std::max(1, (s->key_bits + kRadixBits - 1) / kRadixBits);
}

int blaze_open_hatch(blaze_sim* s) {
  if (!s || s->num_wobj <= 0) return -1;
  CK(cudaStreamSynchronize(s->stream));
  s->num_wobj -= 1;  // Hatch(), GPU_Memory_Transfer.cuh:703-706
  return upload_walls(s);
}

int blaze_set_profile(blaze_sim* s, int on) {
  if (!s) return -1;
  CK(cudaStreamSynchronize(s->stream));
  s->profile = on != 0;
  s->ev_marks.clear();
  s->ev_used = 0;
  return 0;
}

int blaze_profile(blaze_sim* s, float* ms_rebuild, float* ms_step, int* n_steps) {
  if (!s) return -1;
  CK(cudaStreamSynchronize(s->stream));
  float tot[2] = {0.0f, 0.0f};
  int steps = 0;
  for (size_t k = 0; k + 1 < s->ev_marks.size(); k += 2) {
    const int ph = s->ev_marks[k].first;
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, s->ev_pool[s->ev_marks[k].second], s->ev_pool[s->ev_marks[k + 1].second]));
    tot[ph] += ms;
    if (ph == 1) steps++;
  }
  if (ms_rebuild) *ms_rebuild = tot[0];
  if (ms_step) *ms_step = tot[1];
  if (n_steps) *n_steps = steps;
  s->ev_marks.clear();
  s->ev_used = 0;
  return 0;
}

blaze_sim* blaze_default_sim(void) { return g_default; }

// --------------------------------------------- reference interface (Part 1)
namespace {

// The initial lattice Device_Set_SimulationData lays out for a world that
// reads no state file (DeviceInterface.cu:192-707), restated:
//   grid_type 0 (Set_Position_DefaultGrid): num.x x num.y x num.z sites,
//     x fastest then z then y, stepped by p_size[0] + space in FP32 from
//     `start`; types in object order by Num_ParticlesPerObject, P_ID = index;
//     orientations (0, 0, 0, 0) (polyhedra);
//   grid_type 1 (Set_Position_Random_Grid): the same sites; polyhedra get
//     the orientation (30 r1, r2, r3, r4) from four rand() / RAND_MAX each,
//     site by site; types round robin over the objects (an object already
//     at its count gives the site to the first one with room); then N swaps
//     of (type, P_ID) between sites rand() % (N - 1) and rand() % (N - 1).
//     The reference writes the positions of this grid only when particles
//     carry orientations; here every particle gets its site.
// Velocities are InitConfig::velocity[0], spins zero
// (Set_Init_Config_Device, GPU_Memory_Transfer.cuh:214-271).
void initial_lattice(const SimulationInfo& si, const InitConfig& c, int n,
                     std::vector<float3>& pos, std::vector<Quaterion>& q,
                     std::vector<uint>& type, std::vector<int>& pid) {
  pos.assign(n, make_float3(0.0f, 0.0f, 0.0f));
  q.assign(n, Quaterion{0.0f, 0.0f, 0.0f, 0.0f});
  type.assign(n, 0u);
  pid.assign(n, 0);
  const int NX = c.num.x, NY = c.num.y, NZ = c.num.z;
  const float xs = c.p_size[0].x, ys = c.p_size[0].y, zs = c.p_size[0].z;
  const bool orient = si.particle_type == 1 || si.sphere_orient;
  const bool random = c.grid_type == 1;
  const int nobj = std::max(0, std::min(si.Num_ParticleObjects, 6));
  int selectcount[6] = {0, 0, 0, 0, 0, 0};
  int selectT = -1;
  float x = c.start.x, y = c.start.y, z = c.start.z;
  for (int yd = 0; yd < NY; ++yd) {
    for (int zd = 0; zd < NZ; ++zd) {
      for (int xd = 0; xd < NX; ++xd) {
        const int k = yd * NZ * NX + zd * NX + xd;
        if (k < n) {
          pos[k] = make_float3(x, y, z);
          if (random) {
            if (orient) {
              const float rw = ((float)rand() / RAND_MAX) * 30.0;
              const float rx = (float)rand() / RAND_MAX;
              const float ry = (float)rand() / RAND_MAX;
              const float rz = (float)rand() / RAND_MAX;
              q[k] = Quaterion{rw, rx, ry, rz};
            }
            if (++selectT >= nobj) selectT = 0;
            int pty = selectT;
            const int* per = si.Num_ParticlesPerObject;
            if (per && selectcount[pty] >= per[pty]) {
              for (int i = 0; i < nobj; ++i)
                if (selectcount[i] <= per[i] - 1) { pty = i; break; }
            }
            selectcount[pty]++;
            type[k] = (uint)pty;
            pid[k] = k;
          }
        }
        x = x + xs + c.space.x;
      }
      x = c.start.x;
      z = z + zs + c.space.z;
    }
    z = c.start.z;
    y = y + ys + c.space.y;
  }
  if (!random) {
    int idx = 0;
    for (int i = 0; i < si.Num_ParticleObjects && si.Num_ParticlesPerObject; ++i)
      for (int j = 0; j < si.Num_ParticlesPerObject[i] && idx < n; ++j, ++idx) {
        type[idx] = (uint)i;
        pid[idx] = idx;
      }
  } else if (n > 1) {
    for (int i = 0; i < n; ++i) {
      const int src = rand() % (n - 1);
      const int dst = rand() % (n - 1);
      std::swap(type[src], type[dst]);
      std::swap(pid[src], pid[dst]);
    }
  }
}

// Set_Position_Fill_Mill (DeviceInterface.cu:708-1054), restated: the
// whole charge on a lattice of the largest particle's diameter with gaps
// (0.001, 0.001, 0) -- for a ball mill across the drum from its centre
// height upwards (inside the lifters' bound when there are any), else over
// the fill plane -- waves of NX x NZ sites one diameter apart in height;
// types round robin with room, P_ID = site, then the rand() shuffle of
// (type, P_ID); polyhedra get rand() orientations site by site.  Returns
// the wave size; clear = the steps a wave needs to fall two diameters at
// the launch speed.
int fill_lattice(const SimulationInfo& si, const InitConfig& c, const POBJ* po, const WOBJ* w,
                 int n_d, int n, std::vector<float3>& pos, std::vector<Quaterion>& q,
                 std::vector<uint>& type, std::vector<int>& pid, int& clear) {
  pos.assign(n, make_float3(0.0f, 0.0f, 0.0f));
  q.assign(n, Quaterion{0.0f, 0.0f, 0.0f, 0.0f});
  type.assign(n, 0u);
  pid.assign(n, 0);
  const float3 space = make_float3(0.00100f, 0.0010f, 0.0000f);
  const float xs = 2.0 * po[0].radius, ys = 2.0 * po[0].radius, zs = 2.0 * po[0].radius;
  const float radius = n_d > 0 ? si.DObject_CylinderBoundR : w[0].cyl_geo.radius;
  float x, y, z;
  int NX, NY, NZ;
  if (si.Simulation_Type == ballmill && !si.Rotating_WObject) {
    x = n_d > 0 ? xs + (w[0].cyl_geo.radius - si.DObject_CylinderBoundR) : xs + space.x;
    y = w[0].cyl_geo.radius;
    z = w[0].cyl_geo.center_bot_cap.z + zs / 2.0f + space.z;
    NX = (int)floor((radius * 2 - xs) / (xs + space.x));
    NZ = (int)floor((w[0].cyl_geo.height) / (zs + space.z));
    NY = (int)ceil(n / (float)(NX * NZ));
  } else {
    x = c.fill_plane_start.x + xs;
    y = c.fill_plane_start.y;
    z = c.fill_plane_start.z + zs;
    NX = (int)floor((c.fill_plane_end.x - c.fill_plane_start.x) / (xs + space.x));
    NZ = (int)floor((c.fill_plane_end.z - c.fill_plane_start.z) / (zs + space.z));
    NY = (int)ceilf(n / (float)(NX * NZ));
  }
  const float3 start = make_float3(x, y, z);
  clear = (int)fabs((int)ceil((2.0f * ys / (si.InitalDelta_t * c.launch_Vel.y))));
  const bool orient = si.particle_type == 1 || si.sphere_orient;
  const int nobj = std::max(0, std::min(si.Num_ParticleObjects, 6));
  int selectcount[6] = {0, 0, 0, 0, 0, 0};
  int selectT = -1;
  for (int yd = 0; yd < NY; ++yd) {
    for (int zd = 0; zd < NZ; ++zd) {
      for (int xd = 0; xd < NX; ++xd) {
        const int k = yd * NZ * NX + zd * NX + xd;
        if (k >= n) break;
        pos[k] = make_float3(x, y, z);
        if (orient) {
          const float rw = ((float)rand() / RAND_MAX) * 30.0;
          const float rx = (float)rand() / RAND_MAX;
          const float ry = (float)rand() / RAND_MAX;
          const float rz = (float)rand() / RAND_MAX;
          q[k] = Quaterion{rw, rx, ry, rz};
        }
        if (++selectT >= nobj) selectT = 0;
        int pty = selectT;
        const int* per = si.Num_ParticlesPerObject;
        if (per && selectcount[pty] >= per[pty]) {
          for (int i = 0; i < nobj; ++i)
            if (selectcount[i] <= per[i] - 1) { pty = i; break; }
        }
        selectcount[pty]++;
        type[k] = (uint)pty;
        pid[k] = k;
        x = x + xs + space.x;
      }
      x = start.x;
      z = z + zs + space.z;
    }
    z = start.z;
    y = y + ys + space.y;
  }
  for (int i = 0; i < n && n > 1; ++i) {
    const int src = rand() % (n - 1);
    const int dst = rand() % (n - 1);
    std::swap(type[src], type[dst]);
    std::swap(pid[src], pid[dst]);
  }
  return NX * NZ;
}

}  // namespace

int Device_Set_SimulationData(WOBJ* h_WorldOBJ, POBJ* h_ParticleOBJ, DOBJ* h_DynamicOBJ,
                              SimulationInfo* h_SimInfo, int h_Num_WorldOBJ,
                              int h_Num_ParticleOBJ, int h_Num_DynamicOBJ,
                              InitConfig* h_PosConfig) {
  if (g_default) {
    blaze_destroy(g_default);
    g_default = nullptr;
  }
  blaze_sim* s = nullptr;
  int rc = create_impl(&s, h_WorldOBJ, h_Num_WorldOBJ, h_ParticleOBJ, h_Num_ParticleOBJ,
                       h_DynamicOBJ, h_Num_DynamicOBJ, h_SimInfo, nullptr);
  if (rc) return rc;
  g_default = s;
  if (h_PosConfig && !h_PosConfig->use_file) {
    const int n = s->n_max;
    std::vector<float3> pos;
    std::vector<Quaterion> q;
    std::vector<uint> type;
    std::vector<int> pid;
    const bool fill = h_PosConfig->grid_type == 2;
    int clear = 0, pack = 0;
    if (fill)
      pack = fill_lattice(*h_SimInfo, *h_PosConfig, h_ParticleOBJ, h_WorldOBJ, h_Num_DynamicOBJ,
                          n, pos, q, type, pid, clear);
    else
      initial_lattice(*h_SimInfo, *h_PosConfig, n, pos, q, type, pid);
    std::vector<float3> vel(n, h_PosConfig->velocity[0]), avel(n, make_float3(0.0f, 0.0f, 0.0f));
    const bool orient = h_SimInfo->particle_type == 1;
    rc = set_state_impl(s, (const float*)pos.data(), orient ? (const float*)q.data() : nullptr,
                        (const float*)vel.data(), (const float*)avel.data(), type.data(),
                        pid.data());
    if (rc < 0) return rc;
    if (fill && pack > 0) {
      // nothing in the run until the first step's wave (NUMPARTICLES_Current = 0)
      s->filling = true;
      s->fill_n = 0;
      s->fill_pack = pack;
      s->fill_clear = clear;
      s->fill_counter = 0;
      s->h_ctl->n_cur = 0;
      CK(cudaMemcpy(&s->ctl->n_cur, &s->h_ctl->n_cur, sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  return 0;
}

#define DEF_SIM()             \
  blaze_sim* s = g_default;   \
  if (!s) return -2


int Device_Set_Pos(float3* h_pos, Quaterion* h_Ornt, uint* h_ptype, int* h_pid) {
  DEF_SIM();
  return set_state_impl(s, (const float*)h_pos, (const float*)h_Ornt, nullptr, nullptr, h_ptype,
                        h_pid);
}

int Device_Set_Pos_Velocity(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            uint* h_ptype, int* h_pid) {
  DEF_SIM();
  return set_state_impl(s, (const float*)h_pos, (const float*)h_Ornt, (const float*)h_vel,
                        (const float*)h_Avel, h_ptype, h_pid);
}

int Device_Set_System_State(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            float3* h_acc, uint* h_ptype, int* h_pid) {
  (void)h_acc;
  DEF_SIM();
  return set_state_impl(s, (const float*)h_pos, (const float*)h_Ornt, (const float*)h_vel,
                        (const float*)h_Avel, h_ptype, h_pid);
}

int Device_Set_Tallys(float* h_Tallys) {
  DEF_SIM();
  if (!h_Tallys) return -1;
  const double t[3] = {h_Tallys[0], h_Tallys[1], h_Tallys[2]};
  return blaze_set_energy(s, t);
}

int Device_Get_System_State(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            float3* h_acc, uint* h_ptype, int* h_pid) {
  (void)h_acc;
  DEF_SIM();
  int rc = get_state_impl(s, (float*)h_pos, (float*)h_Ornt, (float*)h_vel, (float*)h_Avel, h_ptype,
                          h_pid);
  if (rc >= 0 && h_Ornt && s->si.sphere_orient)
    for (int i = 0; i < s->n_max; ++i) h_Ornt[i] = Quaterion{1.0f, 0.0f, 0.0f, 0.0f};
  return rc;
}

int Device_Get_P_Positions(float3* Pos, Quaterion* Quart_ornt, uint* h_ptype, int* h_pid) {
  DEF_SIM();
  return get_state_impl(s, (float*)Pos, (float*)Quart_ornt, nullptr, nullptr, h_ptype, h_pid);
}

int Device_Get_P_Velocity(float3* H_Vel, float3* H_Rvel, int Flag, uint* h_ptype, int* h_pid) {
  DEF_SIM();
  return get_state_impl(s, nullptr, nullptr, (float*)H_Vel, Flag == 1 ? (float*)H_Rvel : nullptr, h_ptype,
                        h_pid);
}

int Device_Get_W_Forces(float3* WallForces, float3* WallContact_Point) {
  (void)WallContact_Point;
  DEF_SIM();
  if (!WallForces) return -1;
  if (!s->cap_alloc) {
    // wall forces are only materialised when the step keeps its forces
    std::memset(WallForces, 0, sizeof(float3) * s->n_max);
    return -1;
  }
  return blaze_get_forces(s, nullptr, nullptr, (float*)WallForces, nullptr, nullptr, nullptr);
}

int Device_Get_Energy(float* Energy) {
  DEF_SIM();
  if (!Energy) return -1;
  double e[3];
  int rc = blaze_get_energy(s, e);
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) Energy[k] = (float)e[k];
  return 0;
}

int Device_Update_DObjectPostions(DOBJ* h_DynamicOBJ) {
  DEF_SIM();
  return blaze_update_dobj(s, h_DynamicOBJ, s->n_d);
}

int Device_Update_WorldObjectPostions(WOBJ* h_WorldOBJ) {
  DEF_SIM();
  return blaze_update_wobj(s, h_WorldOBJ, s->n_w);
}

int Device_OpenHatch(WOBJ* h_WorldOBJ, int h_Num_WorldOBJ) {
  DEF_SIM();
  if (!h_WorldOBJ || h_Num_WorldOBJ < 0 || h_Num_WorldOBJ > 8) return -1;
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(s->w, h_WorldOBJ, sizeof(WOBJ) * h_Num_WorldOBJ);
  s->num_wobj = s->num_wobj - 1;  // Hatch(): the last world object is dropped
  return upload_walls(s);
}

int Device_Clean(void) {
  if (!g_default) return 0;
  return blaze_destroy(g_default);
}

int Device_Reset_Energy(int num_values) {
  DEF_SIM();
  if (num_values <= 3) return blaze_set_energy(s, nullptr);
  return 0;
}

int drum_rotation(bool cylinder_rotation) {
  DEF_SIM();
  return blaze_set_cylinder_rotation(s, cylinder_rotation ? 1 : 0);
}

int Start_Bin(void) { return 0; }

int Device_AddForce(void) { DEF_SIM(); s->fc += 10.0f; return 0; }
int Device_SubForce(void) { DEF_SIM(); s->fc -= 10.0f; return 0; }
int Device_ZeroForce(void) { DEF_SIM(); s->fc = 0.0f; return 0; }

int Device_DEM_UpdateSim(void) {
  DEF_SIM();
  return blaze_step(s, 1);
}

}  // extern "C"
