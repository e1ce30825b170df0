// ens_capi.cu -- host side of the ensemble path (include/blaze_ens.h): the
// per-system constants, the triangle candidate lists per cell, the buffers
// (allocated once), the step pipeline and its CUDA-graph form.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <utility>
#include <vector>

#include "blaze_dem.h"
#include "blaze_ens.h"
#include "ens_adjoint.cuh"
#include "ens_kernels.cuh"
#include "mix_kernels.cuh"
#include "radix_sort.cuh"

using namespace blaze;

namespace {

int cuda_fail(cudaError_t e) {
  std::fprintf(stderr, "blaze_ens: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
  return -(1000 + (int)e);
}

#define CK(x)                                    \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) return cuda_fail(e_); \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

constexpr int kGraphSteps = 8;

}  // namespace

struct blaze_ens {
  blaze_ens_options opt{};
  int nsys = 0, n = 0, nwalls = 0;
  std::vector<blaze_system> sys;
  std::vector<EnsSysDev> hsys;
  std::vector<EnsWallDev> hwalls;
  EnsSysDev* d_sys = nullptr;
  EnsWallDev* d_walls = nullptr;
  uint32_t* d_tri_off = nullptr;
  uint32_t* d_tri_ids = nullptr;
  uint32_t ncell_tab = 0;
  int key_bits = 1;
  EnsBufs b{};
  int cur = 0;
  RadixSortBuffers rs{};
  uint32_t* cstart = nullptr;
  uint32_t* cend = nullptr;
  StepCtl* ctl = nullptr;
  StepCtl* h_ctl = nullptr;
  int* d_sys_of = nullptr;
  float* st_pos3 = nullptr;   // staging of the caller's arrays
  float* st_rad = nullptr;
  float* st_vel3 = nullptr;
  float* st_avel3 = nullptr;
  int* st_sys = nullptr;
  int* st_pid = nullptr;
  int* d_flags = nullptr;
  int* h_flags = nullptr;
  EnsCapture cap{};
  cudaStream_t stream = nullptr, aux = nullptr, aux2 = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t pgraph[2] = {nullptr, nullptr};   // persistent stepping, home S[c]
  int* d_pw = nullptr;        // persistent stepping: left, done, req_step, barrier x3
  float2* d_rot = nullptr;    // per system: (cos, sin) of the drum's turn so far
  bool any_rot = false;
  int persist_grid = 0;
  int* d_rb = nullptr;
  uint32_t status = 0;
  int last_launches = 0;
  bool state_set = false;
  bool stepped = false;       // a step since the last set_state
  // polyhedra (blaze_ens_set_polyhedra); npoly 0: spheres only
  int npoly = 0, poly_cap = 0, shape_cap = 0;
  MixShapeDev* d_shapes = nullptr;
  float4* d_bv = nullptr;
  double4* d_bn = nullptr;
  uchar4* d_faces = nullptr;
  uchar4* d_edges = nullptr;
  int* d_shape_of = nullptr;
  int* d_pidx = nullptr;
  float4* d_quat = nullptr;
  float4* d_quat0 = nullptr;
  int* d_pat = nullptr;
  float* d_ppath = nullptr;
  double4* d_gv = nullptr;
  double4* d_gf = nullptr;
  float4* d_pwh = nullptr;
  int* d_pwn = nullptr;
  float4* d_psf = nullptr;
  float4* d_pst = nullptr;
  uint8_t* d_twin = nullptr;
  // a finer triangle grid for the spheres of systems with polyhedra (their
  // hash cells are sized for the polyhedra's bounding radii): per system
  // cell, cells and global offset; the CSR lists on it
  std::vector<float> h_rad;               // the radii of the last set_state
  std::vector<float> scell;
  std::vector<int3> snc;
  std::vector<uint32_t> scell_off;
  bool sgrid = false;
  uint32_t* d_stri_off = nullptr;
  uint32_t* d_stri_ids = nullptr;
  MixList ml[2] = {};
  // blaze_ens_set_profile: plain steps timed by phase
  bool prof = false;
  cudaEvent_t pev[5] = {};
  double prof_ms[4] = {0.0, 0.0, 0.0, 0.0};
  int prof_n = 0;
};

namespace {

EnsGeom geom(const blaze_ens* e) {
  EnsGeom g;
  g.sys = e->d_sys;
  g.walls = e->d_walls;
  g.tri_off = e->d_tri_off;
  g.tri_ids = e->d_tri_ids;
  g.stri_off = e->sgrid ? e->d_stri_off : e->d_tri_off;
  g.stri_ids = e->sgrid ? e->d_stri_ids : e->d_tri_ids;
  g.ncell_tab = e->ncell_tab;
  g.law = e->opt.law;
  g.dt = e->opt.dt;
  g.skin = e->opt.skin;
  g.curved = 0;
  for (const EnsWallDev& w : e->hwalls)
    if (w.kind != kWallPlane) g.curved = 1;
  g.rot = e->d_rot;
  g.any_rot = e->any_rot ? 1 : 0;
  g.mix = MixView{};
  if (e->npoly > 0) {
    g.mix.twin = e->d_twin;
    g.mix.sf = e->d_psf;
    g.mix.st = e->d_pst;
    g.mix.npoly = e->npoly;
  }
  return g;
}

MixBufs mix_bufs(const blaze_ens* e) {
  MixBufs m;
  m.shapes = e->d_shapes;
  m.bv = e->d_bv;
  m.bn = e->d_bn;
  m.faces = e->d_faces;
  m.edges = e->d_edges;
  m.shape_of = e->d_shape_of;
  m.quat = e->d_quat;
  m.pat = e->d_pat;
  m.ppath = e->d_ppath;
  m.gv = e->d_gv;
  m.gf = e->d_gf;
  m.wh = e->d_pwh;
  m.wn = e->d_pwn;
  m.sf = e->d_psf;
  m.st = e->d_pst;
  m.twin = e->d_twin;
  m.L[0] = e->ml[0];
  m.L[1] = e->ml[1];
  m.npoly = e->npoly;
  return m;
}

// Per-system constants of the contact law, in double, rounded once to float.
EnsSysDev system_constants(const blaze_system& s, uint32_t cell_off, float dt) {
  EnsSysDev d;
  std::memset(&d, 0, sizeof(d));
  d.origin = make_float3(s.origin[0], s.origin[1], s.origin[2]);
  d.cell = s.cell;
  d.nc = make_int3(s.ncells[0], s.ncells[1], s.ncells[2]);
  d.cell_off = cell_off;
  d.gravity = make_float3(s.gravity[0], s.gravity[1], s.gravity[2]);
  const double pi = 3.14159265358979323846;
  d.dens43pi = (float)((double)s.density * 4.0 / 3.0 * pi);
  const double e = s.restitution;
  const double le = std::log(e);
  const double beta = -le / std::sqrt(le * le + pi * pi);
  d.kn = s.kn;
  d.kt = (float)((double)s.kn * (double)s.kt_ratio);
  d.beta2 = (float)(2.0 * beta);
  const double E = s.youngs, nu = s.poisson;
  d.estar = (float)(E / (2.0 * (1.0 - nu * nu)));
  d.gstar = (float)(E / (4.0 * (2.0 - nu) * (1.0 + nu)));
  d.beta2h = (float)(2.0 * std::sqrt(5.0 / 6.0) * beta);
  d.mu = s.mu;
  d.mu_w = s.mu_wall;
  d.mu_r = s.mu_roll;
  d.wall0 = s.wall0;
  d.nwall = s.nwalls;
  // reference law: Set_SpringConstantsParticleKN / Set_SpringConstantsSurface_KN
  // (KSimulationData.cpp:955-1047): the restitution less 0.03808 inside
  // [0.3, 0.9], Cn = -2 ln(e) sqrt(Kn m) / sqrt(ln(e)^2 + pi^2), none at e = 1
  {
    const double rpi = 2.0 * std::asin(1.0);
    double cor = (double)s.restitution;
    if (cor < 1.0) {
      if (cor >= 0.30 && cor <= 0.90) cor -= 0.038080;
      d.ref_a = -2.0 * std::log(cor);
      d.ref_b = std::sqrt(std::log(cor) * std::log(cor) + rpi * rpi);
    } else {
      d.ref_a = 0.0;
      d.ref_b = 0.0;
    }
    d.ref_m = ((4.0 / 3.0) * rpi) * (double)s.density;
  }
  d.rot_o = make_float3(s.rot_point[0], s.rot_point[1], s.rot_point[2]);
  d.rot_a = make_float3(s.rot_axis[0], s.rot_axis[1], s.rot_axis[2]);
  d.rot_w = s.rot_omega;
  d.rot = s.rot_omega != 0.0f ? 1 : 0;
  {
    const float ang = s.rot_omega * dt;   // the host's single-precision cosine and sine
    d.rot_cd = std::cos(ang);
    d.rot_sd = std::sin(ang);
  }
  d.scell = d.cell;   // the spheres' triangle grid: the hash grid unless blaze_ens::sgrid
  d.snc = d.nc;
  d.scell_off = d.cell_off;
  return d;
}

// A unit vector computed in double from float components.
double3 unit64(double x, double y, double z) {
  const double l = std::sqrt(x * x + y * y + z * z);
  return l > 0 ? make_double3(x / l, y / l, z / l) : make_double3(0.0, 0.0, 0.0);
}

EnsWallDev wall_dev(const blaze_wall& w) {
  EnsWallDev d;
  std::memset(&d, 0, sizeof(d));
  d.kind = w.kind;
  if (w.kind == BLAZE_WALL_PLANE) {
    d.a = make_float3(w.p[0], w.p[1], w.p[2]);
    d.r = w.p[3];
  } else if (w.kind == BLAZE_WALL_TRIANGLE) {
    const float* p = w.p;
    d.a = make_float3(p[0], p[1], p[2]);
    d.b = make_float3(p[3], p[4], p[5]);
    d.c = make_float3(p[6], p[7], p[8]);
    const double ab[3] = {(double)p[3] - p[0], (double)p[4] - p[1], (double)p[5] - p[2]};
    const double ac[3] = {(double)p[6] - p[0], (double)p[7] - p[1], (double)p[8] - p[2]};
    const double bc[3] = {(double)p[6] - p[3], (double)p[7] - p[4], (double)p[8] - p[5]};
    d.n64 = unit64(ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
                   ab[0] * ac[1] - ab[1] * ac[0]);
    d.e64[0] = unit64(ab[0], ab[1], ab[2]);
    d.e64[1] = unit64(ac[0], ac[1], ac[2]);
    d.e64[2] = unit64(bc[0], bc[1], bc[2]);
  } else {
    d.a = make_float3(w.p[0], w.p[1], w.p[2]);
    d.b = make_float3(w.p[3], w.p[4], w.p[5]);
    d.r = w.p[6];
  }
  return d;
}

// Candidate triangles per global cell: every cell whose box meets the
// triangle's bounding box grown by half a cell (more than the largest radius
// a system allows), so a sphere centred in the cell touches no triangle left
// out.  Lists are in ascending triangle order.  spheres_grid: on the spheres'
// finer grid of a system with polyhedra (blaze_ens::scell, half a cell is
// more than any sphere's radius there).
void build_tri_lists(const blaze_ens* e, std::vector<uint32_t>& off, std::vector<uint32_t>& ids,
                     bool spheres_grid = false) {
  uint32_t ntab = e->ncell_tab;
  if (spheres_grid) {
    ntab = 0;
    for (int s = 0; s < e->nsys; ++s)
      ntab += (uint32_t)e->snc[s].x * (uint32_t)e->snc[s].y * (uint32_t)e->snc[s].z;
  }
  off.assign((size_t)ntab + 1, 0);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;  // (cell, triangle)
  for (int s = 0; s < e->nsys; ++s) {
    const blaze_system& S = e->sys[s];
    const EnsSysDev& D = e->hsys[s];
    const float cell = spheres_grid ? e->scell[s] : S.cell;
    const int3 nc = spheres_grid ? e->snc[s] : D.nc;
    const uint32_t coff = spheres_grid ? e->scell_off[s] : D.cell_off;
    const double margin = 0.5 * (double)cell + 1e-4 * (double)cell;
    for (int t = S.tri0; t < S.tri0 + S.ntris; ++t) {
      const EnsWallDev& W = e->hwalls[t];
      const float3 v[3] = {W.a, W.b, W.c};
      int lo[3], hi[3];
      for (int c = 0; c < 3; ++c) {
        double mn = 1e300, mx = -1e300;
        for (int k = 0; k < 3; ++k) {
          const double x = c == 0 ? v[k].x : (c == 1 ? v[k].y : v[k].z);
          mn = std::min(mn, x);
          mx = std::max(mx, x);
        }
        const double o = c == 0 ? D.origin.x : (c == 1 ? D.origin.y : D.origin.z);
        const int ncs = c == 0 ? nc.x : (c == 1 ? nc.y : nc.z);
        lo[c] = std::max(0, (int)std::floor((mn - margin - o) / (double)cell));
        hi[c] = std::min(ncs - 1, (int)std::floor((mx + margin - o) / (double)cell));
      }
      for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
          for (int x = lo[0]; x <= hi[0]; ++x)
            pairs.push_back({coff + (uint32_t)(x + nc.x * (y + nc.y * z)), (uint32_t)t});
    }
  }
  std::stable_sort(pairs.begin(), pairs.end(),
                   [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                     return a.first < b.first;
                   });
  ids.resize(pairs.size());
  for (size_t k = 0; k < pairs.size(); ++k) {
    off[pairs[k].first + 1]++;
    ids[k] = pairs[k].second;
  }
  for (size_t c = 0; c < ntab; ++c) off[c + 1] += off[c];
}

void drop_graphs(blaze_ens* e) {
  for (int c = 0; c < 2; ++c) {
    if (e->graph[c]) cudaGraphExecDestroy(e->graph[c]);
    e->graph[c] = nullptr;
    if (e->pgraph[c]) cudaGraphExecDestroy(e->pgraph[c]);
    e->pgraph[c] = nullptr;
  }
}

void free_ens(blaze_ens* e) {
  if (!e) return;
  drop_graphs(e);
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (int k = 0; k < 3; ++k) { f(e->b.S[k].pos); f(e->b.S[k].vel); f(e->b.S[k].angv); }
  for (int k = 0; k < 2; ++k) {
    f(e->b.pid[k]); f(e->b.wh[k]);
    f(e->b.L[k].idx); f(e->b.L[k].cnt); f(e->b.L[k].mask);
    f(e->b.L[k].hx); f(e->b.L[k].hy); f(e->b.L[k].hz); f(e->b.L[k].src);
    f(e->rs.keys[k]); f(e->rs.vals[k]);
  }
  f(e->rs.counts); f(e->rs.totals); f(e->cstart); f(e->cend); f(e->ctl); f(e->d_rb);
  f(e->d_sys); f(e->d_walls); f(e->d_tri_off); f(e->d_tri_ids); f(e->d_sys_of);
  f(e->st_pos3); f(e->st_rad); f(e->st_vel3); f(e->st_avel3); f(e->st_sys); f(e->st_pid);
  f(e->d_flags); f(e->cap.f); f(e->cap.t); f(e->d_pw); f(e->d_rot);
  f(e->d_shapes); f(e->d_bv); f(e->d_bn); f(e->d_faces); f(e->d_edges); f(e->d_shape_of);
  f(e->d_pidx); f(e->d_quat); f(e->d_quat0); f(e->d_pat); f(e->d_ppath); f(e->d_gv); f(e->d_gf);
  f(e->d_pwh); f(e->d_pwn); f(e->d_psf); f(e->d_pst); f(e->d_twin);
  f(e->d_stri_off); f(e->d_stri_ids);
  for (int k = 0; k < 2; ++k) {
    f(e->ml[k].idx); f(e->ml[k].cnt); f(e->ml[k].mlo); f(e->ml[k].mhi);
    f(e->ml[k].hx); f(e->ml[k].hy); f(e->ml[k].hz); f(e->ml[k].sep);
  }
  if (e->h_ctl) cudaFreeHost(e->h_ctl);
  for (int k = 0; k < 5; ++k)
    if (e->pev[k]) cudaEventDestroy(e->pev[k]);
  if (e->h_flags) cudaFreeHost(e->h_flags);
  if (e->aux2) cudaStreamDestroy(e->aux2);
  if (e->aux) cudaStreamDestroy(e->aux);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

bool valid_system(const blaze_system& s, int nwalls, float skin) {
  if (s.n < 0 || !(s.cell > 0.0f) || s.ncells[0] < 1 || s.ncells[1] < 1 || s.ncells[2] < 1)
    return false;
  if (!(s.cell >= skin)) return false;
  if (!(s.density > 0.0f) || !(s.restitution > 0.0f) || !(s.restitution <= 1.0f)) return false;
  if (s.wall0 < 0 || s.nwalls < 0 || s.wall0 + s.nwalls > nwalls) return false;
  if (s.tri0 < 0 || s.ntris < 0 || s.tri0 + s.ntris > nwalls) return false;
  if (!std::isfinite(s.rot_omega)) return false;
  if (s.rot_omega != 0.0f) {
    const double ax = s.rot_axis[0], ay = s.rot_axis[1], az = s.rot_axis[2];
    if (!(std::fabs(std::sqrt(ax * ax + ay * ay + az * az) - 1.0) < 1e-5)) return false;
  }
  return true;
}

int upload_params(blaze_ens* e) {
  uint32_t off = 0;
  e->hsys.resize(e->nsys);
  for (int s = 0; s < e->nsys; ++s) {
    e->hsys[s] = system_constants(e->sys[s], off, e->opt.dt);
    off += (uint32_t)e->sys[s].ncells[0] * (uint32_t)e->sys[s].ncells[1] *
           (uint32_t)e->sys[s].ncells[2];
    if (e->sgrid) {
      e->hsys[s].scell = e->scell[s];
      e->hsys[s].snc = e->snc[s];
      e->hsys[s].scell_off = e->scell_off[s];
    }
  }
  CK(cudaMemcpyAsync(e->d_sys, e->hsys.data(), sizeof(EnsSysDev) * e->nsys,
                     cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return 0;
}

int enqueue_rebuild(blaze_ens* e, const int* gate, cudaStream_t st) {
  const int n = e->n;
  const EnsGeom g = geom(e);
  ens_launch_hash(g, e->b, e->cur, n, e->rs.keys[0], e->ctl, gate, st);
  const int res = radix_sort_pairs(e->rs, n, e->key_bits, true, gate, st);
  CK(cudaMemsetAsync(e->cstart, 0xff, sizeof(uint32_t) * e->ncell_tab, st));
  ens_launch_reorder(e->b, e->cur, n, e->rs.keys[res], e->rs.vals[res], e->cstart, e->cend,
                     e->ncell_tab, e->ctl, gate, st);
  ens_launch_nlist(g, e->b, n, e->rs.vals[res], e->cstart, e->cend, e->ctl, gate, st);
  if (e->npoly > 0) {
    mix_launch_plist(g, e->b, mix_bufs(e), e->cstart, e->cend, e->ctl, gate, st);
    mix_launch_twins(e->b, mix_bufs(e), n, e->ctl, gate, st);
  }
  ens_launch_epoch(e->ctl, gate, st);
  return 0;
}

int rebuild_kernel_count(const blaze_ens* e) {
  return 4 + 3 * std::max(1, (e->key_bits + kRadixBits - 1) / kRadixBits) + (e->npoly > 0 ? 2 : 0);
}

// The step's kernels: polyhedron geometry, the sphere step, the polyhedron
// step (the last two read the same input state and write disjoint entries).
// The step's kernels: polyhedron geometry, the polyhedron step (which leaves
// the sphere-polyhedron pairs' forces on the spheres), the sphere step; the
// last two read the same input state and write disjoint entries.  ev
// (profiling, or null): recorded after each of the three.
void launch_step_kernels(blaze_ens* e, StepLink link, cudaStream_t st,
                         const cudaEvent_t* ev = nullptr) {
  const EnsCapture* cap = e->opt.capture_forces ? &e->cap : nullptr;
  if (e->npoly > 0) mix_launch_geom(mix_bufs(e), st);
  if (ev) cudaEventRecord(ev[0], st);
  if (e->npoly > 0) mix_launch_poly_step(geom(e), e->b, mix_bufs(e), e->cur, e->ctl, link, cap, st);
  if (ev) cudaEventRecord(ev[1], st);
  ens_launch_step(geom(e), e->b, e->cur, e->n, e->ctl, link, cap, e->opt.block, st);
  if (ev) cudaEventRecord(ev[2], st);
}

int step_kernel_count(const blaze_ens* e) {
  return 1 + (e->npoly > 0 ? 2 : 0) + (e->any_rot ? 1 : 0);
}

int enqueue_step(blaze_ens* e) {
  if (e->prof) CK(cudaEventRecord(e->pev[0], e->stream));
  launch_gate(e->ctl, e->stream);
  int rc = enqueue_rebuild(e, &e->ctl->rebuilt, e->stream);
  if (rc) return rc;
  if (e->prof) CK(cudaEventRecord(e->pev[1], e->stream));
  launch_step_kernels(e, StepLink{&e->ctl->rebuilt, 0, 0}, e->stream, e->prof ? e->pev + 2 : nullptr);
  if (e->any_rot) ens_launch_rot_tick(geom(e), e->nsys, e->stream);
  e->last_launches += 1 + step_kernel_count(e) + rebuild_kernel_count(e);
  e->cur ^= 1;
  if (e->prof) {   // re-sort, polyhedron geometry, polyhedron step, sphere step
    CK(cudaEventSynchronize(e->pev[4]));
    for (int k = 0; k < 4; ++k) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, e->pev[k], e->pev[k + 1]));
      e->prof_ms[k] += ms;
    }
    e->prof_n += 1;
  }
  return 0;
}

// kGraphSteps steps as one graph starting from S[c]: a gate kernel carries
// the pending re-sort request into the first step's IF node; each step kernel
// sets the next step's IF condition when any particle has moved half the skin.
int build_graph(blaze_ens* e, int c) {
  const int saved = e->cur;
  e->cur = c;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h[kGraphSteps];
  for (int k = 0; k < kGraphSteps; ++k)
    CK(cudaGraphConditionalHandleCreate(&h[k], g, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(e->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  launch_gate_graph(e->ctl, h[0], e->d_rb, kGraphSteps, e->stream);
  for (int k = 0; k < kGraphSteps; ++k) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(e->stream, &cs, nullptr, &capg, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h[k];
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(e->stream, &cnode, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(e->aux, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    CK(cudaMemsetAsync(e->d_rb + k, 0x01, sizeof(int), e->aux));
    int rc = enqueue_rebuild(e, nullptr, e->aux);
    cudaGraph_t tmp = nullptr;
    CK(cudaStreamEndCapture(e->aux, &tmp));
    if (rc) return rc;
    const StepLink link = k + 1 < kGraphSteps ? StepLink{e->d_rb + k, h[k + 1], 1}
                                               : StepLink{e->d_rb + k, 0, 0};
    launch_step_kernels(e, link, e->stream);
    if (e->any_rot) ens_launch_rot_tick(geom(e), e->nsys, e->stream);
    e->cur ^= 1;
  }
  cudaGraph_t out = nullptr;
  CK(cudaStreamEndCapture(e->stream, &out));
  CK(cudaGraphInstantiate(&e->graph[c], out, 0));
  CK(cudaGraphDestroy(out));
  e->cur = saved;
  return 0;
}

EnsPersist persist_words(const blaze_ens* e, cudaGraphConditionalHandle loop_h) {
  EnsPersist p;
  p.left = e->d_pw;
  p.done = e->d_pw + 1;
  p.req_step = e->d_pw + 2;
  p.bar = reinterpret_cast<unsigned int*>(e->d_pw + 4);
  p.loop_h = loop_h;
  return p;
}

// Persistent stepping from and back to S[c]: one graph whose WHILE node runs
// rounds until the step budget (*left, set before each launch) is spent.  A
// round is a gate kernel (pending re-sort request into the IF node), the IF
// node with the re-sort, and the persistent step kernel, which runs steps
// until one asks for a re-sort or the budget is spent.
int build_persist_graph_as(blaze_ens* e, int c, bool coop) {
  if (e->persist_grid <= 0) {
    e->persist_grid = ens_persist_grid(geom(e), e->opt.block, e->n);
    if (e->persist_grid <= 0) return -2;
  }
  const int saved = e->cur;
  e->cur = c;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hw;
  CK(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault));
  const EnsPersist p = persist_words(e, hw);
  CK(cudaStreamBeginCaptureToGraph(e->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  {
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(e->stream, &cs, nullptr, &capg, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hw;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, capg, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(e->stream, &wnode, 1, cudaStreamSetCaptureDependencies));
    // the round, captured into the loop body on aux
    cudaGraphConditionalHandle hi;
    CK(cudaGraphConditionalHandleCreate(&hi, body, 0, 0));
    CK(cudaStreamBeginCaptureToGraph(e->aux, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    ens_launch_persist_gate(e->ctl, p, e->d_rb, hi, e->aux);
    {
      cudaStreamCaptureStatus cs2;
      cudaGraph_t capb = nullptr;
      const cudaGraphNode_t* deps2 = nullptr;
      size_t ndeps2 = 0;
      CK(cudaStreamGetCaptureInfo(e->aux, &cs2, nullptr, &capb, &deps2, &ndeps2));
      alignas(cudaGraphNodeParams) unsigned char raw2[sizeof(cudaGraphNodeParams)];
      std::memset(raw2, 0, sizeof(raw2));
      cudaGraphNodeParams& ip = *reinterpret_cast<cudaGraphNodeParams*>(raw2);
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = hi;
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t inode;
      CK(cudaGraphAddNode(&inode, capb, deps2, ndeps2, &ip));
      cudaGraph_t ibody = ip.conditional.phGraph_out[0];
      CK(cudaStreamUpdateCaptureDependencies(e->aux, &inode, 1, cudaStreamSetCaptureDependencies));
      CK(cudaStreamBeginCaptureToGraph(e->aux2, ibody, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal));
      CK(cudaMemsetAsync(e->d_rb, 0x01, sizeof(int), e->aux2));
      rc = enqueue_rebuild(e, nullptr, e->aux2);
      cudaGraph_t tmp = nullptr;
      CK(cudaStreamEndCapture(e->aux2, &tmp));
    }
    cudaError_t le = cudaSuccess;
    if (!rc)
      le = ens_launch_persist(geom(e), e->b, c, e->n, e->ctl, e->d_rb, p, e->opt.block,
                              e->persist_grid, coop, e->aux);
    cudaGraph_t tmp = nullptr;
    cudaError_t ee = cudaStreamEndCapture(e->aux, &tmp);
    if (!rc && (le != cudaSuccess || ee != cudaSuccess)) rc = -3;
  }
  cudaGraph_t out = nullptr;
  cudaError_t ee = cudaStreamEndCapture(e->stream, &out);
  if (!rc && ee != cudaSuccess) rc = -3;
  if (!rc && cudaGraphInstantiate(&e->pgraph[c], out, 0) != cudaSuccess) rc = -3;
  if (out) cudaGraphDestroy(out);
  e->cur = saved;
  return rc;
}

// A cooperative kernel node guarantees that every block of the persistent
// kernel is resident; where a conditional body does not take one, the
// kernel node is a plain one with the same occupancy-sized grid (the
// barrier's bounded wait turns a block that could not start into
// kStatusTimeout, not a hang).
int build_persist_graph(blaze_ens* e, int c) {
  int rc = build_persist_graph_as(e, c, true);
  if (rc == -3) {
    cudaGetLastError();
    rc = build_persist_graph_as(e, c, false);
  }
  if (rc == -3) {
    cudaGetLastError();
    return -1;
  }
  return rc;
}

int sync_status(blaze_ens* e) {
  CK(cudaMemcpyAsync(e->h_ctl, e->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  CK(cudaGetLastError());
  e->status |= e->h_ctl->status;
  return (int)e->status;
}

int create_impl(blaze_ens** out, const blaze_system* systems, int nsys, const blaze_wall* walls,
                int nwalls, const blaze_ens_options* opt) {
  if (!out || !systems || nsys < 1 || nsys > (int)kSysMask || nwalls < 0 || (nwalls && !walls))
    return -1;
  blaze_ens_options o;
  if (opt) o = *opt;
  else blaze_ens_default_options(&o);
  if ((o.law != BLAZE_LAW_LINEAR && o.law != BLAZE_LAW_HERTZ_MINDLIN &&
       o.law != BLAZE_LAW_REFERENCE) || !(o.dt > 0.0f) ||
      !(o.skin > 0.0f) || o.max_nbr < 1 || o.max_nbr > 32)
    return -1;
  if (o.block == 0) o.block = 256;
  if (o.block < 64 || o.block > kMaxStepBlock || o.block % 32 != 0) return -1;
  if (o.use_graph < 0 || o.use_graph > 2) return -1;
  long long ntot = 0, cells = 0;
  for (int s = 0; s < nsys; ++s) {
    if (!valid_system(systems[s], nwalls, o.skin)) return -1;
    ntot += systems[s].n;
    cells += (long long)systems[s].ncells[0] * systems[s].ncells[1] * systems[s].ncells[2];
  }
  for (int w = 0; w < nwalls; ++w)
    if (walls[w].kind < BLAZE_WALL_PLANE || walls[w].kind > BLAZE_WALL_CYLINDER) return -1;
  for (int s = 0; s < nsys; ++s) {
    // the reference law meets plane walls only
    if (o.law == BLAZE_LAW_REFERENCE && (systems[s].ntris > 0 || systems[s].rot_omega != 0.0f))
      return -1;
    for (int w = systems[s].wall0; w < systems[s].wall0 + systems[s].nwalls; ++w) {
      if (walls[w].kind == BLAZE_WALL_TRIANGLE) return -1;
      if (o.law == BLAZE_LAW_REFERENCE && walls[w].kind != BLAZE_WALL_PLANE) return -1;
    }
    for (int w = systems[s].tri0; w < systems[s].tri0 + systems[s].ntris; ++w)
      if (walls[w].kind != BLAZE_WALL_TRIANGLE) return -1;
  }
  if (ntot < 1 || ntot > (1ll << 30) || cells + 1 >= (1ll << 32)) return -1;

  blaze_ens* e = new (std::nothrow) blaze_ens();
  if (!e) return -1;
  auto fail = [&](int rc) { free_ens(e); return rc; };
#define CKF(x) do { cudaError_t e2 = (x); if (e2 != cudaSuccess) return fail(cuda_fail(e2)); } while (0)
  e->opt = o;
  e->nsys = nsys;
  e->n = (int)ntot;
  e->nwalls = nwalls;
  e->sys.assign(systems, systems + nsys);
  e->ncell_tab = (uint32_t)cells;
  for (int w = 0; w < nwalls; ++w) e->hwalls.push_back(wall_dev(walls[w]));
  // walls that turn in place with a drum: cylinders coaxial with it, planes
  // normal to its axis (their surfaces move; their positions do not)
  for (int s = 0; s < nsys; ++s) {
    const blaze_system& y = systems[s];
    if (y.rot_omega == 0.0f) continue;
    const double ax = y.rot_axis[0], ay = y.rot_axis[1], az = y.rot_axis[2];
    for (int w = y.wall0; w < y.wall0 + y.nwalls; ++w) {
      EnsWallDev& W = e->hwalls[w];
      const double a[3] = {W.a.x, W.a.y, W.a.z}, b[3] = {W.b.x, W.b.y, W.b.z};
      if (W.kind == kWallPlane) {
        W.turning = std::fabs(std::fabs(a[0] * ax + a[1] * ay + a[2] * az) - 1.0) < 1e-6 ? 1 : 0;
      } else if (W.kind == kWallCylinder) {
        // axis parallel, and the axis point on the turn's axis
        const double par = std::fabs(b[0] * ax + b[1] * ay + b[2] * az);
        const double d[3] = {a[0] - y.rot_point[0], a[1] - y.rot_point[1], a[2] - y.rot_point[2]};
        const double dd = d[0] * ax + d[1] * ay + d[2] * az;
        const double off = std::sqrt(std::max(0.0, d[0] * d[0] + d[1] * d[1] + d[2] * d[2] - dd * dd));
        W.turning = (std::fabs(par - 1.0) < 1e-6 && off < 1e-4) ? 1 : 0;
      }
    }
  }
  const uint32_t top = e->ncell_tab + 1u;
  e->key_bits = 1;
  while (e->key_bits < 32 && (top >> e->key_bits) != 0) e->key_bits++;
  CKF(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  CKF(cudaStreamCreateWithFlags(&e->aux, cudaStreamNonBlocking));
  CKF(cudaStreamCreateWithFlags(&e->aux2, cudaStreamNonBlocking));
  const int n = e->n;
  const int cap = o.max_nbr;
  e->b.stride = n;
  e->b.cap = cap;
  for (int k = 0; k < 3; ++k) {
    CKF(dalloc(&e->b.S[k].pos, n)); CKF(dalloc(&e->b.S[k].vel, n)); CKF(dalloc(&e->b.S[k].angv, n));
  }
  for (int k = 0; k < 2; ++k) {
    CKF(dalloc(&e->b.pid[k], n));
    CKF(dalloc(&e->b.wh[k], (size_t)kWallSlots * n));
    CKF(dalloc(&e->b.L[k].idx, (size_t)cap * n));
    CKF(dalloc(&e->b.L[k].cnt, n));
    CKF(dalloc(&e->b.L[k].mask, n));
    CKF(dalloc(&e->b.L[k].hx, (size_t)cap * n));
    CKF(dalloc(&e->b.L[k].hy, (size_t)cap * n));
    CKF(dalloc(&e->b.L[k].hz, (size_t)cap * n));
    CKF(dalloc(&e->b.L[k].src, (size_t)cap * n));
    CKF(dalloc(&e->rs.keys[k], n));
    CKF(dalloc(&e->rs.vals[k], n));
    CKF(cudaMemset(e->b.L[k].cnt, 0, sizeof(uint32_t) * n));
    CKF(cudaMemset(e->b.L[k].mask, 0, sizeof(uint32_t) * n));
  }
  const int tiles = (n + kTileKeys - 1) / kTileKeys;
  e->rs.max_n = n;
  e->rs.max_tiles = tiles;
  CKF(dalloc(&e->rs.counts, (size_t)kRadixDigits * std::max(tiles, 1)));
  CKF(dalloc(&e->rs.totals, kRadixDigits));
  CKF(dalloc(&e->cstart, e->ncell_tab));
  CKF(dalloc(&e->cend, e->ncell_tab));
  CKF(dalloc(&e->ctl, 1));
  CKF(dalloc(&e->d_rb, kGraphSteps));
  CKF(cudaMemset(e->d_rb, 0, sizeof(int) * kGraphSteps));
  CKF(dalloc(&e->d_pw, 8));
  CKF(cudaMemset(e->d_pw, 0, sizeof(int) * 8));
  CKF(dalloc(&e->d_rot, nsys));
  for (int s = 0; s < nsys; ++s) e->any_rot = e->any_rot || systems[s].rot_omega != 0.0f;
  {
    const std::vector<float2> id((size_t)nsys, make_float2(1.0f, 0.0f));
    CKF(cudaMemcpy(e->d_rot, id.data(), sizeof(float2) * nsys, cudaMemcpyHostToDevice));
  }
  CKF(dalloc(&e->d_sys, nsys));
  CKF(dalloc(&e->d_walls, nwalls));
  CKF(dalloc(&e->d_sys_of, n));
  CKF(dalloc(&e->st_pos3, (size_t)3 * n));
  CKF(dalloc(&e->st_rad, n));
  CKF(dalloc(&e->st_vel3, (size_t)3 * n));
  CKF(dalloc(&e->st_avel3, (size_t)3 * n));
  CKF(dalloc(&e->st_sys, n));
  CKF(dalloc(&e->st_pid, n));
  CKF(dalloc(&e->d_flags, 2));
  CKF(cudaMallocHost((void**)&e->h_flags, 2 * sizeof(int)));
  CKF(cudaMallocHost((void**)&e->h_ctl, sizeof(StepCtl)));
  if (o.capture_forces) {
    CKF(dalloc(&e->cap.f, n));
    CKF(dalloc(&e->cap.t, n));
    CKF(cudaMemset(e->cap.f, 0, sizeof(float4) * n));
    CKF(cudaMemset(e->cap.t, 0, sizeof(float4) * n));
  }
  for (int k = 0; k < 3; ++k) {
    CKF(cudaMemset(e->b.S[k].pos, 0, sizeof(float4) * n));
    CKF(cudaMemset(e->b.S[k].vel, 0, sizeof(float4) * n));
    CKF(cudaMemset(e->b.S[k].angv, 0, sizeof(float4) * n));
  }
  {
    std::vector<int> so(n);
    int k = 0;
    for (int s = 0; s < nsys; ++s)
      for (int q = 0; q < systems[s].n; ++q) so[k++] = s;
    CKF(cudaMemcpy(e->d_sys_of, so.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  }
  if (nwalls)
    CKF(cudaMemcpy(e->d_walls, e->hwalls.data(), sizeof(EnsWallDev) * nwalls,
                   cudaMemcpyHostToDevice));
  int rc = upload_params(e);
  if (rc) return fail(rc);
  bool any_tri = false;
  for (int s = 0; s < nsys; ++s) any_tri = any_tri || systems[s].ntris > 0;
  if (any_tri) {
    std::vector<uint32_t> off, ids;
    build_tri_lists(e, off, ids);
    CKF(dalloc(&e->d_tri_off, off.size()));
    CKF(dalloc(&e->d_tri_ids, ids.size()));
    CKF(cudaMemcpy(e->d_tri_off, off.data(), sizeof(uint32_t) * off.size(), cudaMemcpyHostToDevice));
    if (!ids.empty())
      CKF(cudaMemcpy(e->d_tri_ids, ids.data(), sizeof(uint32_t) * ids.size(), cudaMemcpyHostToDevice));
  }
  std::memset(e->h_ctl, 0, sizeof(StepCtl));
  e->h_ctl->n_cur = n;
  e->h_ctl->rebuild_req = 1;
  CKF(cudaMemcpy(e->ctl, e->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice));
  CKF(cudaDeviceSynchronize());
#undef CKF
  *out = e;
  return 0;
}

}  // namespace

extern "C" {

void blaze_ens_default_options(blaze_ens_options* o) {
  if (!o) return;
  o->law = BLAZE_LAW_LINEAR;
  o->dt = 1e-5f;
  o->skin = 0.02f;
  o->max_nbr = 32;
  o->use_graph = 1;
  o->capture_forces = 0;
  o->block = 256;
}

int blaze_ens_create(blaze_ens** out, const blaze_system* systems, int nsys,
                     const blaze_wall* walls, int nwalls, const blaze_ens_options* opt) {
  return create_impl(out, systems, nsys, walls, nwalls, opt);
}

int blaze_ens_destroy(blaze_ens* e) {
  if (!e) return -1;
  cudaStreamSynchronize(e->stream);
  free_ens(e);
  return 0;
}

int blaze_ens_set_state(blaze_ens* e, const float* pos3, const float* radius, const float* vel3,
                        const float* avel3) {
  if (!e || !pos3 || !radius) return -1;
  const int n = e->n;
  // every radius must fit its system's cell: 2 r + skin <= cell
  {
    int k = 0;
    for (int s = 0; s < e->nsys; ++s) {
      const float lim = 0.5f * (e->sys[s].cell - e->opt.skin);
      for (int q = 0; q < e->sys[s].n; ++q, ++k)
        if (!(radius[k] > 0.0f) || radius[k] > lim) return -1;
    }
  }
  int rc = sync_status(e);
  if (rc < 0) return rc;
  e->h_rad.assign(radius, radius + n);
  CK(cudaMemsetAsync(e->d_flags, 0, 2 * sizeof(int), e->stream));
  CK(cudaMemcpyAsync(e->st_pos3, pos3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(e->st_rad, radius, sizeof(float) * n, cudaMemcpyHostToDevice, e->stream));
  if (vel3)
    CK(cudaMemcpyAsync(e->st_vel3, vel3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, e->stream));
  if (avel3)
    CK(cudaMemcpyAsync(e->st_avel3, avel3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, e->stream));
  const int ep = e->h_ctl->epoch & 1;
  ens_launch_pack(e->st_pos3, e->st_rad, vel3 ? e->st_vel3 : nullptr, avel3 ? e->st_avel3 : nullptr,
                  e->d_sys_of, e->b, e->cur, e->b.pid[ep], n, e->d_flags, e->stream);
  if (e->any_rot) {   // the drums start from the walls' given positions
    const std::vector<float2> id((size_t)e->nsys, make_float2(1.0f, 0.0f));
    CK(cudaMemcpyAsync(e->d_rot, id.data(), sizeof(float2) * e->nsys, cudaMemcpyHostToDevice,
                       e->stream));
  }
  CK(cudaMemcpyAsync(e->h_flags, e->d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  CK(cudaGetLastError());
  if (e->h_flags[0]) return -1;
  StepCtl c = *e->h_ctl;
  c.rebuild_req = 1;
  c.rebuilt = 0;
  c.status = 0;
  c.n_cur = n;
  c.pending_dead = 0;
  *e->h_ctl = c;
  e->status = 0;
  CK(cudaMemcpyAsync(e->ctl, e->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->state_set = true;
  e->stepped = false;
  if (e->npoly > 0) {   // spheres only again: the graphs hold the polyhedron kernels
    e->npoly = 0;
    e->b.pat = nullptr;
    e->b.ppath = nullptr;
    drop_graphs(e);
  }
  if (e->sgrid) {       // the spheres' triangles on the hash grid again
    e->sgrid = false;
    int rp = upload_params(e);
    if (rp) return rp;
  }
  return 0;
}

int blaze_ens_get_state(blaze_ens* e, float* pos3, float* radius, float* vel3, float* avel3,
                        int* sys, int* pid) {
  if (!e) return -1;
  int st = sync_status(e);
  if (st < 0) return st;
  const int n = e->n;
  const int ep = e->h_ctl->epoch & 1;
  ens_launch_unpack(e->b, e->cur, n, e->b.pid[ep], e->st_pos3, e->st_rad, e->st_vel3, e->st_avel3,
                    e->st_sys, e->st_pid, e->stream);
  if (pos3) CK(cudaMemcpyAsync(pos3, e->st_pos3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, e->stream));
  if (radius) CK(cudaMemcpyAsync(radius, e->st_rad, sizeof(float) * n, cudaMemcpyDeviceToHost, e->stream));
  if (vel3) CK(cudaMemcpyAsync(vel3, e->st_vel3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, e->stream));
  if (avel3) CK(cudaMemcpyAsync(avel3, e->st_avel3, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, e->stream));
  if (sys) CK(cudaMemcpyAsync(sys, e->st_sys, sizeof(int) * n, cudaMemcpyDeviceToHost, e->stream));
  if (pid) CK(cudaMemcpyAsync(pid, e->st_pid, sizeof(int) * n, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  CK(cudaGetLastError());
  return st;
}

}  // extern "C"

namespace {

// nsteps steps, as kGraphSteps-step CUDA graphs where `graphs` allows (the
// remainder as plain steps).
int advance(blaze_ens* e, int nsteps, bool graphs) {
  // persistent stepping (no drum turns: those advance between steps)
  if (graphs && e->opt.use_graph == 2 && !e->opt.capture_forces && !e->any_rot && e->npoly == 0 &&
      nsteps > 0) {
    const int c = e->cur;
    if (!e->pgraph[c]) {
      int rc = build_persist_graph(e, c);
      if (rc) return rc;
    }
    ens_launch_persist_init(persist_words(e, 0), nsteps, e->stream);
    CK(cudaGraphLaunch(e->pgraph[c], e->stream));
    e->last_launches += 3;   // the budget, then one round's gate and step kernels
    return 0;
  }
  int done = 0;
  while (done < nsteps) {
    if (!graphs || nsteps - done < kGraphSteps) {
      int rc = enqueue_step(e);
      if (rc) return rc;
      done += 1;
      continue;
    }
    const int c = e->cur;
    if (!e->graph[c]) {
      int rc = build_graph(e, c);
      if (rc) return rc;
    }
    CK(cudaGraphLaunch(e->graph[c], e->stream));
    e->last_launches += 1 + kGraphSteps * step_kernel_count(e);
    if (kGraphSteps & 1) e->cur ^= 1;
    done += kGraphSteps;
  }
  CK(cudaGetLastError());
  return 0;
}

}  // namespace

extern "C" {

int blaze_ens_check_barrier_timeout(void) {
  unsigned int* bar = nullptr;
  StepCtl* ctl = nullptr;
  if (cudaMalloc((void**)&bar, 4 * sizeof(unsigned int)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&ctl, sizeof(StepCtl)) != cudaSuccess) {
    cudaFree(bar);
    return -1;
  }
  cudaMemset(bar, 0, 4 * sizeof(unsigned int));
  cudaMemset(ctl, 0, sizeof(StepCtl));
  ens_launch_barrier_check(bar, ctl, 0);
  StepCtl h;
  const cudaError_t e = cudaMemcpy(&h, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost);
  cudaFree(bar);
  cudaFree(ctl);
  return e == cudaSuccess ? (int)h.status : -(1000 + (int)e);
}

int blaze_ens_step(blaze_ens* e, int nsteps) {
  if (!e || nsteps < 0 || !e->state_set) return -1;
  e->last_launches = 0;
  if (nsteps > 0) e->stepped = true;
  return advance(e, nsteps, e->opt.use_graph != 0 && !e->prof);
}

int blaze_ens_set_profile(blaze_ens* e, int on) {
  if (!e) return -1;
  if (on && !e->pev[0])
    for (int k = 0; k < 5; ++k) CK(cudaEventCreate(&e->pev[k]));
  e->prof = on != 0;
  for (int k = 0; k < 4; ++k) e->prof_ms[k] = 0.0;
  e->prof_n = 0;
  return 0;
}

int blaze_ens_profile(blaze_ens* e, float* ms4, int* steps) {
  if (!e || !ms4) return -1;
  for (int k = 0; k < 4; ++k) ms4[k] = (float)e->prof_ms[k];
  if (steps) *steps = e->prof_n;
  return 0;
}

int blaze_ens_sync(blaze_ens* e) {
  if (!e) return -1;
  return sync_status(e);
}

int blaze_ens_set_params(blaze_ens* e, const blaze_system* systems) {
  if (!e || !systems) return -1;
  for (int s = 0; s < e->nsys; ++s) {
    const blaze_system& a = e->sys[s];
    const blaze_system& b = systems[s];
    if (b.n != a.n || b.cell != a.cell || b.ncells[0] != a.ncells[0] || b.ncells[1] != a.ncells[1] ||
        b.ncells[2] != a.ncells[2] || b.origin[0] != a.origin[0] || b.origin[1] != a.origin[1] ||
        b.origin[2] != a.origin[2] || b.wall0 != a.wall0 || b.nwalls != a.nwalls ||
        b.tri0 != a.tri0 || b.ntris != a.ntris || !valid_system(b, e->nwalls, e->opt.skin))
      return -1;
  }
  CK(cudaStreamSynchronize(e->stream));
  e->sys.assign(systems, systems + e->nsys);
  return upload_params(e);
}

int blaze_ens_get_forces(blaze_ens* e, float* force3, float* torque3) {
  if (!e || !e->opt.capture_forces) return -1;
  int st = sync_status(e);
  if (st < 0) return st;
  const int n = e->n;
  std::vector<float4> f(n), t(n);
  CK(cudaMemcpy(f.data(), e->cap.f, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(t.data(), e->cap.t, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) {
    if (force3) { force3[3 * i] = f[i].x; force3[3 * i + 1] = f[i].y; force3[3 * i + 2] = f[i].z; }
    if (torque3) { torque3[3 * i] = t[i].x; torque3[3 * i + 1] = t[i].y; torque3[3 * i + 2] = t[i].z; }
  }
  return st;
}

int blaze_ens_num_rebuilds(blaze_ens* e) {
  if (!e) return -1;
  int rc = sync_status(e);
  if (rc < 0) return rc;
  return e->h_ctl->epoch;
}

int blaze_ens_device_state(blaze_ens* e, void** pos4, void** vel4, void** angv4, void** stream) {
  if (!e) return -1;
  if (pos4) *pos4 = e->b.S[e->cur].pos;
  if (vel4) *vel4 = e->b.S[e->cur].vel;
  if (angv4) *angv4 = e->b.S[e->cur].angv;
  if (stream) *stream = (void*)e->stream;
  return 0;
}

int blaze_ens_last_launches(blaze_ens* e) { return e ? e->last_launches : -1; }

int blaze_ens_rebuild_kernels(blaze_ens* e) {
  if (!e) return -1;
  // persistent stepping: a re-sort also starts another round (gate + step)
  return rebuild_kernel_count(e) + (e->opt.use_graph == 2 ? 2 : 0);
}

}  // extern "C"

// ============================================================== polyhedra
namespace {

struct ShapeHost {
  MixShapeDev dev;
  float4 bv[kMixMaxV];
  double4 bn[kMixMaxF];
  uchar4 faces[kMixMaxF];
  uchar4 edges[kMixMaxE];
  double mass, com[3], J[9], rb;
};

// A closed, outward-oriented convex hull of triangles (every directed edge
// once, its reverse once; V - E + F = 2; every vertex on or below every face
// plane), its unit face normals, its edges (vertex i < j, in (i, j) order,
// faces f1 < f2) and its mass properties, in FP64: volume, centre of mass
// and inertia from the tetrahedra of the faces with the origin
// (covariance of a tetrahedron (0, a, b, c): det / 120 (a a^T + b b^T +
// c c^T + s s^T), s = a + b + c; inertia = tr(C) 1 - C, moved to the centre
// of mass).
bool shape_setup(const blaze_shape& s, ShapeHost& o) {
  std::memset(&o, 0, sizeof(o));
  const int nv = s.nverts, nf = s.nfaces;
  if (nv < 4 || nv > kMixMaxV || nf != 2 * nv - 4 || !(s.density > 0.0f) ||
      !std::isfinite(s.density))
    return false;
  double v[kMixMaxV][3];
  for (int k = 0; k < nv; ++k)
    for (int c = 0; c < 3; ++c) {
      if (!std::isfinite(s.verts[3 * k + c])) return false;
      v[k][c] = (double)s.verts[3 * k + c];
    }
  std::map<std::pair<int, int>, int> dir;
  for (int f = 0; f < nf; ++f) {
    const int a = s.faces[3 * f], b = s.faces[3 * f + 1], c = s.faces[3 * f + 2];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv || a == b || b == c || a == c)
      return false;
    const int ed[3][2] = {{a, b}, {b, c}, {c, a}};
    for (int k = 0; k < 3; ++k) {
      const std::pair<int, int> key(ed[k][0], ed[k][1]);
      if (dir.count(key)) return false;
      dir[key] = f;
    }
    o.faces[f] = make_uchar4((unsigned char)a, (unsigned char)b, (unsigned char)c, 0);
    const double e1[3] = {v[b][0] - v[a][0], v[b][1] - v[a][1], v[b][2] - v[a][2]};
    const double e2[3] = {v[c][0] - v[a][0], v[c][1] - v[a][1], v[c][2] - v[a][2]};
    const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                          e1[0] * e2[1] - e1[1] * e2[0]};
    const double l = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    if (!(l > 0.0)) return false;
    o.bn[f] = make_double4(cr[0] / l, cr[1] / l, cr[2] / l, 0.0);
  }
  int ne = 0;
  for (const auto& kv : dir) {
    const int a = kv.first.first, b = kv.first.second;
    const auto rev = dir.find(std::make_pair(b, a));
    if (rev == dir.end()) return false;
    if (a > b) continue;
    if (ne >= kMixMaxE) return false;
    const int f1 = std::min(kv.second, rev->second), f2 = std::max(kv.second, rev->second);
    o.edges[ne++] = make_uchar4((unsigned char)a, (unsigned char)b, (unsigned char)f1,
                                (unsigned char)f2);
  }
  if (ne != 3 * nv - 6 || nv - ne + nf != 2) return false;
  double rb = 0.0;
  for (int k = 0; k < nv; ++k)
    rb = std::max(rb, std::sqrt(v[k][0] * v[k][0] + v[k][1] * v[k][1] + v[k][2] * v[k][2]));
  for (int f = 0; f < nf; ++f) {
    const double* n = &o.bn[f].x;
    const double* p0 = v[o.faces[f].x];
    const double h = n[0] * p0[0] + n[1] * p0[1] + n[2] * p0[2];
    for (int k = 0; k < nv; ++k)
      if (n[0] * v[k][0] + n[1] * v[k][1] + n[2] * v[k][2] - h > 1e-6 * rb) return false;
  }
  double vol = 0.0, cen[3] = {0.0, 0.0, 0.0}, C[9] = {0.0};
  for (int f = 0; f < nf; ++f) {
    const double* a = v[o.faces[f].x];
    const double* b = v[o.faces[f].y];
    const double* c = v[o.faces[f].z];
    const double det = a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
                       a[2] * (b[0] * c[1] - b[1] * c[0]);
    vol += det / 6.0;
    double sm[3];
    for (int q = 0; q < 3; ++q) {
      sm[q] = a[q] + b[q] + c[q];
      cen[q] += det * sm[q] / 24.0;
    }
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        C[3 * r + q] += det / 120.0 * (a[r] * a[q] + b[r] * b[q] + c[r] * c[q] + sm[r] * sm[q]);
  }
  if (!(vol > 0.0)) return false;
  const double rho = (double)s.density;
  o.mass = rho * vol;
  for (int q = 0; q < 3; ++q) o.com[q] = cen[q] / vol;
  const double tr = C[0] + C[4] + C[8];
  const double c2 = o.com[0] * o.com[0] + o.com[1] * o.com[1] + o.com[2] * o.com[2];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q)
      o.J[3 * r + q] = rho * ((r == q ? tr : 0.0) - C[3 * r + q]) -
                       o.mass * ((r == q ? c2 : 0.0) - o.com[r] * o.com[q]);
  const double* J = o.J;
  const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]);
  if (!(det > 0.0)) return false;
  const double inv[9] = {(J[4] * J[8] - J[5] * J[7]) / det, (J[2] * J[7] - J[1] * J[8]) / det,
                         (J[1] * J[5] - J[2] * J[4]) / det, (J[5] * J[6] - J[3] * J[8]) / det,
                         (J[0] * J[8] - J[2] * J[6]) / det, (J[2] * J[3] - J[0] * J[5]) / det,
                         (J[3] * J[7] - J[4] * J[6]) / det, (J[1] * J[6] - J[0] * J[7]) / det,
                         (J[0] * J[4] - J[1] * J[3]) / det};
  o.rb = rb;
  float rbf = (float)rb;
  if ((double)rbf < rb) rbf = std::nextafter(rbf, INFINITY);
  o.dev.nv = nv;
  o.dev.nf = nf;
  o.dev.ne = ne;
  o.dev.mass = (float)o.mass;
  o.dev.rb = rbf;
  for (int q = 0; q < 9; ++q) {
    o.dev.inertia[q] = (float)J[q];
    o.dev.iinv[q] = (float)inv[q];
  }
  for (int k = 0; k < nv; ++k)
    o.bv[k] = make_float4(s.verts[3 * k], s.verts[3 * k + 1], s.verts[3 * k + 2], 0.0f);
  return true;
}

// A device array of `count` elements in place of the old one.
template <class T>
int realloc_dev(T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  CK(dalloc(p, count));
  return 0;
}

}  // namespace

extern "C" {

int blaze_shape_mass_properties(const blaze_shape* s, double* mass, double* com3,
                                double* inertia9, float* rbound) {
  if (!s) return -1;
  ShapeHost h;
  if (!shape_setup(*s, h)) return -1;
  if (mass) *mass = h.mass;
  if (com3)
    for (int q = 0; q < 3; ++q) com3[q] = h.com[q];
  if (inertia9)
    for (int q = 0; q < 9; ++q) inertia9[q] = h.J[q];
  if (rbound) *rbound = h.dev.rb;
  return 0;
}

int blaze_ens_set_polyhedra(blaze_ens* e, const blaze_shape* shapes, int nshapes,
                            const int* shape_of, const float* quat4) {
  if (!e || !shapes || nshapes < 1 || !shape_of || !quat4) return -1;
  if (!e->state_set || e->stepped || e->opt.law != BLAZE_LAW_LINEAR) return -1;
  std::vector<ShapeHost> hs(nshapes);
  for (int k = 0; k < nshapes; ++k) {
    if (!shape_setup(shapes[k], hs[k])) return -1;
    const double* c = hs[k].com;
    if (std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) > 1e-4 * hs[k].rb) return -1;
  }
  std::vector<int> pidx, pshape;
  std::vector<float4> q0;
  int i = 0;
  for (int sy = 0; sy < e->nsys; ++sy) {
    const blaze_system& S = e->sys[sy];
    for (int k = 0; k < S.n; ++k, ++i) {
      const int sh = shape_of[i];
      if (sh < 0) continue;
      if (sh >= nshapes) return -1;
      if (2.0f * hs[sh].dev.rb + e->opt.skin > S.cell) return -1;
      for (int w = S.wall0; w < S.wall0 + S.nwalls; ++w)
        if (e->hwalls[w].kind != kWallPlane) return -1;
      const double qw = quat4[4 * i], qx = quat4[4 * i + 1], qy = quat4[4 * i + 2],
                   qz = quat4[4 * i + 3];
      const double qn = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
      if (!(qn > 0.0) || !std::isfinite(qn)) return -1;
      pidx.push_back(i);
      pshape.push_back(sh);
      q0.push_back(make_float4((float)(qw / qn), (float)(qx / qn), (float)(qy / qn),
                               (float)(qz / qn)));
    }
  }
  int rc = sync_status(e);
  if (rc < 0) return rc;
  const int np = (int)pidx.size();
  drop_graphs(e);
  e->npoly = 0;
  e->b.pat = nullptr;
  e->b.ppath = nullptr;
  if (np == 0) return 0;
  if (nshapes > e->shape_cap) {
    if ((rc = realloc_dev(&e->d_shapes, (size_t)nshapes)) || (rc = realloc_dev(&e->d_bv, (size_t)nshapes * kMixMaxV)) ||
        (rc = realloc_dev(&e->d_bn, (size_t)nshapes * kMixMaxF)) ||
        (rc = realloc_dev(&e->d_faces, (size_t)nshapes * kMixMaxF)) ||
        (rc = realloc_dev(&e->d_edges, (size_t)nshapes * kMixMaxE)))
      return rc;
    e->shape_cap = nshapes;
  }
  if (np > e->poly_cap) {
    if ((rc = realloc_dev(&e->d_shape_of, (size_t)np)) || (rc = realloc_dev(&e->d_pidx, (size_t)np)) ||
        (rc = realloc_dev(&e->d_quat, (size_t)np)) || (rc = realloc_dev(&e->d_quat0, (size_t)np)) ||
        (rc = realloc_dev(&e->d_pat, (size_t)np)) || (rc = realloc_dev(&e->d_ppath, (size_t)np)) ||
        (rc = realloc_dev(&e->d_gv, (size_t)np * kMixMaxV)) ||
        (rc = realloc_dev(&e->d_gf, (size_t)np * kMixMaxF)) ||
        (rc = realloc_dev(&e->d_pwh, (size_t)np * kMixWallSlots)) ||
        (rc = realloc_dev(&e->d_pwn, (size_t)np)) ||
        (rc = realloc_dev(&e->d_psf, (size_t)np * kMixSlots)) ||
        (rc = realloc_dev(&e->d_pst, (size_t)np * kMixSlots)))
      return rc;
    for (int k = 0; k < 2; ++k) {
      MixList& L = e->ml[k];
      if ((rc = realloc_dev(&L.idx, (size_t)np * kMixSlots)) || (rc = realloc_dev(&L.cnt, (size_t)np)) ||
          (rc = realloc_dev(&L.mlo, (size_t)np)) || (rc = realloc_dev(&L.mhi, (size_t)np)) ||
          (rc = realloc_dev(&L.hx, (size_t)np * kMixSlots)) || (rc = realloc_dev(&L.hy, (size_t)np * kMixSlots)) ||
          (rc = realloc_dev(&L.hz, (size_t)np * kMixSlots)) ||
          (rc = realloc_dev(&L.sep, (size_t)np * kMixSlots)))
        return rc;
    }
    e->poly_cap = np;
  }
  if (!e->d_twin && (rc = realloc_dev(&e->d_twin, (size_t)e->b.cap * e->n))) return rc;
  // the spheres' triangles on a grid of cells of 2 r_max(spheres) + skin
  // where that is finer than the hash grid (sized for the polyhedra)
  {
    bool any = false;
    e->scell.assign(e->nsys, 0.0f);
    e->snc.assign(e->nsys, make_int3(0, 0, 0));
    e->scell_off.assign(e->nsys, 0u);
    uint32_t off = 0;
    int i0 = 0;
    for (int sy = 0; sy < e->nsys; ++sy) {
      const blaze_system& S = e->sys[sy];
      float rmax = 0.0f;
      bool has_poly = false;
      for (int k = 0; k < S.n; ++k) {
        if (shape_of[i0 + k] >= 0) has_poly = true;
        else rmax = std::max(rmax, e->h_rad[i0 + k]);
      }
      i0 += S.n;
      const float fine = (2.0f * rmax + e->opt.skin) * (1.0f + 1e-6f);
      if (has_poly && S.ntris > 0 && rmax > 0.0f && fine < 0.8f * S.cell) {
        e->scell[sy] = fine;
        for (int c = 0; c < 3; ++c) {
          const int m = (int)std::ceil((double)S.ncells[c] * (double)S.cell / (double)fine);
          (c == 0 ? e->snc[sy].x : (c == 1 ? e->snc[sy].y : e->snc[sy].z)) = m;
        }
        any = true;
      } else {
        e->scell[sy] = S.cell;
        e->snc[sy] = make_int3(S.ncells[0], S.ncells[1], S.ncells[2]);
      }
      e->scell_off[sy] = off;
      off += (uint32_t)e->snc[sy].x * (uint32_t)e->snc[sy].y * (uint32_t)e->snc[sy].z;
    }
    if (any) {
      std::vector<uint32_t> off_v, ids;
      build_tri_lists(e, off_v, ids, true);
      if ((rc = realloc_dev(&e->d_stri_off, off_v.size())) ||
          (rc = realloc_dev(&e->d_stri_ids, std::max<size_t>(ids.size(), 1))))
        return rc;
      CK(cudaMemcpy(e->d_stri_off, off_v.data(), sizeof(uint32_t) * off_v.size(),
                    cudaMemcpyHostToDevice));
      if (!ids.empty())
        CK(cudaMemcpy(e->d_stri_ids, ids.data(), sizeof(uint32_t) * ids.size(),
                      cudaMemcpyHostToDevice));
    }
    e->sgrid = any;
    if ((rc = upload_params(e))) return rc;
  }
  {
    std::vector<MixShapeDev> sd(nshapes);
    std::vector<float4> bv((size_t)nshapes * kMixMaxV, make_float4(0, 0, 0, 0));
    std::vector<double4> bn((size_t)nshapes * kMixMaxF, make_double4(0, 0, 0, 0));
    std::vector<uchar4> fa((size_t)nshapes * kMixMaxF, make_uchar4(0, 0, 0, 0));
    std::vector<uchar4> ed((size_t)nshapes * kMixMaxE, make_uchar4(0, 0, 0, 0));
    for (int k = 0; k < nshapes; ++k) {
      sd[k] = hs[k].dev;
      std::copy(hs[k].bv, hs[k].bv + kMixMaxV, bv.begin() + (size_t)k * kMixMaxV);
      std::copy(hs[k].bn, hs[k].bn + kMixMaxF, bn.begin() + (size_t)k * kMixMaxF);
      std::copy(hs[k].faces, hs[k].faces + kMixMaxF, fa.begin() + (size_t)k * kMixMaxF);
      std::copy(hs[k].edges, hs[k].edges + kMixMaxE, ed.begin() + (size_t)k * kMixMaxE);
    }
    CK(cudaMemcpy(e->d_shapes, sd.data(), sizeof(MixShapeDev) * nshapes, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_bv, bv.data(), sizeof(float4) * bv.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_bn, bn.data(), sizeof(double4) * bn.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_faces, fa.data(), sizeof(uchar4) * fa.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_edges, ed.data(), sizeof(uchar4) * ed.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(e->d_shape_of, pshape.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->d_pidx, pidx.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->d_quat0, q0.data(), sizeof(float4) * np, cudaMemcpyHostToDevice));
  CK(cudaMemset(e->d_gv, 0, sizeof(double4) * (size_t)np * kMixMaxV));
  CK(cudaMemset(e->d_gf, 0, sizeof(double4) * (size_t)np * kMixMaxF));
  e->npoly = np;
  e->b.pat = e->d_pat;
  e->b.ppath = e->d_ppath;
  mix_launch_mark(e->b, e->cur, mix_bufs(e), e->d_pidx, e->d_quat0, e->stream);
  CK(cudaStreamSynchronize(e->stream));
  CK(cudaGetLastError());
  return 0;
}

int blaze_ens_get_orientations(blaze_ens* e, float* quat4) {
  if (!e || !quat4) return -1;
  int st = sync_status(e);
  if (st < 0) return st;
  const int n = e->n;
  std::vector<float4> pos(n), angv(n), q(std::max(e->npoly, 1));
  CK(cudaMemcpy(pos.data(), e->b.S[e->cur].pos, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(angv.data(), e->b.S[e->cur].angv, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  if (e->npoly > 0)
    CK(cudaMemcpy(q.data(), e->d_quat, sizeof(float4) * e->npoly, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) {
    float4 o = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
    if (e->npoly > 0 && pos[i].w < 0.0f) {
      int p;
      std::memcpy(&p, &angv[i].w, sizeof(int));
      if (p >= 0 && p < e->npoly) o = q[p];
    }
    quat4[4 * i] = o.x;
    quat4[4 * i + 1] = o.y;
    quat4[4 * i + 2] = o.z;
    quat4[4 * i + 3] = o.w;
  }
  return st;
}

}  // extern "C"

// ============================================================ reverse mode
struct EnsCheckpoint {
  float4* pos = nullptr;
  float4* vel = nullptr;
  float4* angv = nullptr;
  int* pid = nullptr;
  uint32_t* idx = nullptr;
  uint32_t* cnt = nullptr;
  uint32_t* mask = nullptr;
  float* hx = nullptr;
  float* hy = nullptr;
  float* hz = nullptr;
  float4* wh = nullptr;
  StepCtl ctl{};
  int cur = 0;
};

// Where a recorded segment lies in the tape arena: words [o, e).  `valid`
// while nothing recorded later overlapped them and its own reservations all
// fit.
struct TapeSeg {
  unsigned long long o = 0, e = 0;
  bool valid = false;
  std::vector<int> rb;          // per step: 1 when it re-sorted
};

struct blaze_ens_adj {
  blaze_ens* e = nullptr;
  int nsteps = 0, K = 0, nseg = 0;
  EnsTape tape{};
  unsigned long long words = 0;            // arena size
  unsigned long long stride = 0;           // dense block of one step, words
  TapeCtl* h_tc = nullptr;                 // pinned copy of the tape cursors
  std::vector<TapeStep> h_steps;           // staging for the re-sort flags
  std::vector<EnsCheckpoint> ck;
  std::vector<TapeSeg> seg;
  int on_tape = 0;                         // segments the last forward left on the tape
  unsigned long long pool_max = 0;         // most pool words one recorded segment took
  double pool_step = 0.0;                  // most pool words per step of a segment
  AdjBufs A{};
  bool forward_done = false;
  cudaGraphExec_t rgraph[2] = {nullptr, nullptr};  // recording graphs, from S[0] / S[1]
  // per-phase device time of the last backward call (restoring checkpoints,
  // recording segments into the tape, reversing them), from events
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  float ms_phase[3] = {0.0f, 0.0f, 0.0f};
  int* d_sys_off = nullptr;     // nsys + 1 particle offsets of the systems
  double* d_gconst = nullptr;   // 5 per system: summed law-constant cotangents
};

namespace {

int sort_result(const blaze_ens* e) {
  const int passes = std::max(1, (e->key_bits + kRadixBits - 1) / kRadixBits);
  return passes & 1;
}

void free_adj(blaze_ens_adj* a) {
  if (!a) return;
  for (cudaEvent_t ev : a->ev)
    if (ev) cudaEventDestroy(ev);
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(a->tape.arena);
  f(a->tape.steps);
  f(a->tape.ctl);
  if (a->h_tc) cudaFreeHost(a->h_tc);
  for (EnsCheckpoint& c : a->ck) {
    f(c.pos); f(c.vel); f(c.angv); f(c.pid); f(c.idx); f(c.cnt); f(c.mask); f(c.hx); f(c.hy);
    f(c.hz); f(c.wh);
  }
  AdjBufs& b = a->A;
  for (float4* q : {b.gx, b.gv, b.gw, b.gH, b.gW, b.ix, b.iv, b.iw, b.iH, b.iW, b.Fb, b.px,
                    b.pv, b.pw})
    f(q);
  f(b.th);
  f(a->d_sys_off);
  f(a->d_gconst);
  for (int c = 0; c < 2; ++c)
    if (a->rgraph[c]) cudaGraphExecDestroy(a->rgraph[c]);
  delete a;
}

int save_checkpoint(blaze_ens_adj* a, EnsCheckpoint& c) {
  blaze_ens* e = a->e;
  int rc = sync_status(e);
  if (rc < 0) return rc;
  const size_t n = e->n, cn = (size_t)e->opt.max_nbr * n;
  const int ep = e->h_ctl->epoch & 1;
  const EnsList& L = e->b.L[ep];
  cudaStream_t st = e->stream;
  CK(cudaMemcpyAsync(c.pos, e->b.S[e->cur].pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.vel, e->b.S[e->cur].vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.angv, e->b.S[e->cur].angv, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.pid, e->b.pid[ep], sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.idx, L.idx, sizeof(uint32_t) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.cnt, L.cnt, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.mask, L.mask, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.hx, L.hx, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.hy, L.hy, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.hz, L.hz, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(c.wh, e->b.wh[ep], sizeof(float4) * kWallSlots * n, cudaMemcpyDeviceToDevice, st));
  c.ctl = *e->h_ctl;
  c.cur = e->cur;
  return 0;
}

int restore_checkpoint(blaze_ens_adj* a, const EnsCheckpoint& c) {
  blaze_ens* e = a->e;
  const size_t n = e->n, cn = (size_t)e->opt.max_nbr * n;
  const int ep = c.ctl.epoch & 1;
  const EnsList& L = e->b.L[ep];
  cudaStream_t st = e->stream;
  e->cur = c.cur;
  CK(cudaMemcpyAsync(e->b.S[e->cur].pos, c.pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(e->b.S[e->cur].vel, c.vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(e->b.S[e->cur].angv, c.angv, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(e->b.pid[ep], c.pid, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.idx, c.idx, sizeof(uint32_t) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.cnt, c.cnt, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.mask, c.mask, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.hx, c.hx, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.hy, c.hy, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(L.hz, c.hz, sizeof(float) * cn, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(e->b.wh[ep], c.wh, sizeof(float4) * kWallSlots * n, cudaMemcpyDeviceToDevice, st));
  *e->h_ctl = c.ctl;
  CK(cudaMemcpyAsync(e->ctl, e->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

// kGraphSteps recorded steps as one graph from S[c]: the step graph of
// build_graph, with the list recorded inside each step's IF node (a
// re-sort), then the tape tick and the recording step.
int build_record_graph(blaze_ens_adj* a, int c) {
  blaze_ens* e = a->e;
  const int res = sort_result(e);
  const int saved = e->cur;
  e->cur = c;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h[kGraphSteps];
  for (int k = 0; k < kGraphSteps; ++k)
    CK(cudaGraphConditionalHandleCreate(&h[k], g, 0, cudaGraphCondAssignDefault));
  CK(cudaStreamBeginCaptureToGraph(e->stream, g, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  launch_gate_graph(e->ctl, h[0], e->d_rb, kGraphSteps, e->stream);
  for (int k = 0; k < kGraphSteps; ++k) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(e->stream, &cs, nullptr, &capg, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h[k];
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, capg, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(e->stream, &cnode, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(e->aux, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    CK(cudaMemsetAsync(e->d_rb + k, 0x01, sizeof(int), e->aux));
    int rc = enqueue_rebuild(e, nullptr, e->aux);
    adj_launch_list(e->b, a->tape, e->n, e->ctl, nullptr, 1, e->rs.vals[res], e->aux);
    cudaGraph_t tmp = nullptr;
    CK(cudaStreamEndCapture(e->aux, &tmp));
    if (rc) return rc;
    adj_launch_tick(a->tape, e->d_rb + k, e->stream);
    const StepLink link = k + 1 < kGraphSteps ? StepLink{e->d_rb + k, h[k + 1], 1}
                                               : StepLink{e->d_rb + k, 0, 0};
    ens_launch_step_record(geom(e), e->b, e->cur, e->n, e->ctl, link, a->tape, e->opt.block,
                           e->stream);
    e->cur ^= 1;
  }
  cudaGraph_t out = nullptr;
  CK(cudaStreamEndCapture(e->stream, &out));
  CK(cudaGraphInstantiate(&a->rgraph[c], out, 0));
  CK(cudaGraphDestroy(out));
  e->cur = saved;
  return 0;
}

// Steps the ensemble through segment `s` from its current state, recording
// it into the arena from word `origin` (dense blocks, then pool space up to
// `lim`).  Fills `sg`; sg.valid is false when a reservation did not fit.
int record_segment(blaze_ens_adj* a, int s, unsigned long long origin, unsigned long long lim,
                   TapeSeg& sg) {
  blaze_ens* e = a->e;
  const int res = sort_result(e);
  const int slot0 = s * a->K, len = std::min(a->K, a->nsteps - slot0);
  cudaStream_t st = e->stream;
  adj_launch_seg_start(a->tape, slot0, len, origin, a->stride, lim, st);
  adj_launch_list(e->b, a->tape, e->n, e->ctl, nullptr, 0, nullptr, st);   // the current list
  int t = 0;
  while (t < len) {
    if (len - t >= kGraphSteps) {
      const int c = e->cur;
      if (!a->rgraph[c]) {
        int rc = build_record_graph(a, c);
        if (rc) return rc;
      }
      CK(cudaGraphLaunch(a->rgraph[c], st));
      if (kGraphSteps & 1) e->cur ^= 1;
      t += kGraphSteps;
      continue;
    }
    launch_gate(e->ctl, st);
    int rc = enqueue_rebuild(e, &e->ctl->rebuilt, st);
    if (rc) return rc;
    adj_launch_list(e->b, a->tape, e->n, e->ctl, &e->ctl->rebuilt, 1, e->rs.vals[res], st);
    adj_launch_tick(a->tape, &e->ctl->rebuilt, st);
    ens_launch_step_record(geom(e), e->b, e->cur, e->n, e->ctl, StepLink{&e->ctl->rebuilt, 0, 0},
                           a->tape, e->opt.block, st);
    e->cur ^= 1;
    ++t;
  }
  CK(cudaMemcpyAsync(a->h_steps.data(), a->tape.steps + slot0, sizeof(TapeStep) * len,
                     cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(a->h_tc, a->tape.ctl, sizeof(TapeCtl), cudaMemcpyDeviceToHost, st));
  int rc = sync_status(e);
  if (rc < 0) return rc;
  sg.rb.assign(len, 0);
  for (int q = 0; q < len; ++q) sg.rb[q] = a->h_steps[q].rb;
  sg.o = origin;
  sg.e = std::min(a->h_tc->cur, lim);
  sg.valid = a->h_tc->overflow == 0;
  if (sg.valid) {
    const unsigned long long pool = sg.e - origin - (unsigned long long)len * a->stride;
    a->pool_max = std::max(a->pool_max, pool);
    a->pool_step = std::max(a->pool_step, (double)pool / len);
  }
  return 0;
}

bool overlaps(const TapeSeg& x, const TapeSeg& y) { return x.o < y.e && y.o < x.e; }

}  // namespace

extern "C" {

int blaze_ens_adj_create_tape(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment,
                              unsigned long long arena_bytes) {
  if (!out || !e || nsteps < 1 || segment < 1 || e->npoly > 0) return -1;
  const unsigned long long aw = arena_bytes / 4 & ~3ull;
  if (aw < (unsigned long long)std::min(segment, nsteps) * tape_block_words(e->n)) return -2;
  if (e->opt.law != BLAZE_LAW_LINEAR || e->any_rot) return -1;
  for (const blaze_system& s : e->sys)
    if (s.mu_roll > 0.0f || s.ntris > 0) return -1;
  for (const EnsWallDev& w : e->hwalls)
    if (w.kind != kWallPlane) return -1;
  blaze_ens_adj* a = new (std::nothrow) blaze_ens_adj();
  if (!a) return -1;
  auto fail = [&](int rc) { free_adj(a); return rc; };
#define CKA(x) do { cudaError_t e2 = (x); if (e2 != cudaSuccess) return fail(cuda_fail(e2)); } while (0)
  a->e = e;
  a->nsteps = nsteps;
  a->K = std::min(segment, nsteps);
  a->nseg = (nsteps + a->K - 1) / a->K;
  a->seg.resize(a->nseg);
  const size_t n = e->n, cap = e->opt.max_nbr, K = a->K;
  a->ck.resize(a->nseg);
  for (EnsCheckpoint& c : a->ck) {
    CKA(dalloc(&c.pos, n)); CKA(dalloc(&c.vel, n)); CKA(dalloc(&c.angv, n)); CKA(dalloc(&c.pid, n));
    CKA(dalloc(&c.idx, cap * n)); CKA(dalloc(&c.cnt, n)); CKA(dalloc(&c.mask, n));
    CKA(dalloc(&c.hx, cap * n)); CKA(dalloc(&c.hy, cap * n)); CKA(dalloc(&c.hz, cap * n));
    CKA(dalloc(&c.wh, kWallSlots * n));
  }
  AdjBufs& b = a->A;
  for (float4** q : {&b.gx, &b.gv, &b.gw, &b.ix, &b.iv, &b.iw}) CKA(dalloc(q, n));
  CKA(dalloc(&b.px, cap * n));
  CKA(dalloc(&b.pv, cap * n));
  CKA(dalloc(&b.pw, cap * n));
  CKA(dalloc(&b.gH, cap * n));
  CKA(dalloc(&b.iH, cap * n));
  CKA(dalloc(&b.gW, kWallSlots * n));
  CKA(dalloc(&b.iW, kWallSlots * n));
  CKA(dalloc(&b.th, 5 * n));
  CKA(dalloc(&b.Fb, n));   // host cotangent stage (12 B of every 16 used)
  CKA(dalloc(&a->d_sys_off, e->nsys + 1));
  CKA(dalloc(&a->d_gconst, 5 * (size_t)e->nsys));
  {
    std::vector<int> off(e->nsys + 1, 0);
    for (int s = 0; s < e->nsys; ++s) off[s + 1] = off[s] + e->sys[s].n;
    CKA(cudaMemcpy(a->d_sys_off, off.data(), sizeof(int) * (e->nsys + 1),
                   cudaMemcpyHostToDevice));
  }
  // the tape: the arena and one step record per step of the run
  a->words = aw;
  a->stride = tape_block_words(e->n);
  a->h_steps.resize(a->K);
  CKA(dalloc(&a->tape.arena, (size_t)aw));
  CKA(dalloc(&a->tape.steps, (size_t)nsteps));
  CKA(dalloc(&a->tape.ctl, 1));
  CKA(cudaMallocHost((void**)&a->h_tc, sizeof(TapeCtl)));
#undef CKA
  *out = a;
  return 0;
}

int blaze_ens_adj_create_ex(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment,
                            long long tape_bytes) {
  if (!out || !e || nsteps < 1 || segment < 1) return -1;
  const size_t n = e->n, cap = e->opt.max_nbr, K = (size_t)std::min(segment, nsteps);
  if (tape_bytes == 0) {
    // one segment with the most pool space it can take: every list slot an
    // active history, every wall slot used, a list at every step
    const size_t words = K * tape_block_words(e->n) + K * n * (3 * cap + 4 * kWallSlots) +
                         (K + 1) * (n * 2 * cap + 256);
    return blaze_ens_adj_create_tape(out, e, nsteps, segment, 4ull * (words + 64));
  }
  size_t budget;
  if (tape_bytes > 0) {
    budget = (size_t)tape_bytes;
  } else {
    // what the other buffers of the reverse mode leave free: all device
    // memory but 4 GiB, less 4 %
    const int nseg = (nsteps + (int)K - 1) / (int)K;
    const size_t ckpt = n * (3 * sizeof(float4) + 3 * sizeof(uint32_t) + sizeof(int) +
                             kWallSlots * sizeof(float4)) + cap * n * 4 * sizeof(float);
    const size_t bufs = n * (7 * sizeof(float4) + 5 * sizeof(float) +
                             2 * kWallSlots * sizeof(float4)) + cap * n * 5 * sizeof(float4);
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    const size_t other = ckpt * (size_t)nseg + bufs + ((size_t)4 << 30);
    budget = fr > other ? (fr - other) / 100 * 96 : 0;
  }
  return blaze_ens_adj_create_tape(out, e, nsteps, segment, (unsigned long long)budget);
}

int blaze_ens_adj_create(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment) {
  return blaze_ens_adj_create_ex(out, e, nsteps, segment, 0);
}

int blaze_ens_adj_forward(blaze_ens_adj* a) {
  if (!a || !a->e->state_set) return -1;
  blaze_ens* e = a->e;
  // the trailing segments expected to fit (dense blocks, plus the most pool
  // space per step seen so far) are recorded as they run (recording graphs);
  // the others run as plain step graphs between checkpoints.  Graph and
  // plain stepping give the same results, so a later recomputation
  // reproduces this run exactly.
  const double per_step = (double)a->stride + a->pool_step;
  auto seg_len = [&](int s) { return std::min(a->K, a->nsteps - s * a->K); };
  int first = a->nseg;
  for (double need = 0.0; first > 0; --first) {
    need += per_step * seg_len(first - 1);
    if (need > (double)a->words) break;
  }
  unsigned long long pos = 0;
  for (TapeSeg& sg : a->seg) sg.valid = false;
  for (int s = 0; s < a->nseg; ++s) {
    int rc = save_checkpoint(a, a->ck[s]);
    if (rc) return rc;
    const int len = seg_len(s);
    if (s < first) {
      rc = advance(e, len, true);
      if (rc) return rc;
      continue;
    }
    // a ring of segments in the arena: wrap to its start when the segment is
    // not expected to fit before the end
    if ((double)pos + per_step * len > (double)a->words) pos = 0;
    TapeSeg& sg = a->seg[s];
    rc = record_segment(a, s, pos, a->words, sg);
    if (rc) return rc;
    for (int r = first; r < s; ++r)
      if (a->seg[r].valid && overlaps(a->seg[r], sg)) a->seg[r].valid = false;
    pos = sg.valid ? (sg.e + 3) & ~3ull : a->words;
  }
  int st = sync_status(e);
  if (st < 0) return st;
  a->on_tape = 0;
  for (const TapeSeg& sg : a->seg) a->on_tape += sg.valid ? 1 : 0;
  a->forward_done = true;
  return st;
}

namespace {

// The reverse sweep over steps [first, nsteps): first = 0 is the whole run;
// first > 0 the window of the last nsteps - first steps.
int backward_impl(blaze_ens_adj* a, int first, const float* gpos, const float* gvel,
                  const float* gavel, float* gpos0, float* gvel0, float* gavel0,
                  double* gconst) {
  if (!a || !a->forward_done || first < 0 || first >= a->nsteps) return -1;
  blaze_ens* e = a->e;
  const size_t n = e->n, cap = e->opt.max_nbr;
  cudaStream_t st = e->stream;
  AdjBufs& A = a->A;
  {
    // host cotangents through a device stage (A.Fb, 16 B per particle,
    // holds the 12 B of one array)
    float* stage = reinterpret_cast<float*>(A.Fb);
    const float* src[3] = {gpos, gvel, gavel};
    float4* dst[3] = {A.gx, A.gv, A.gw};
    for (int q = 0; q < 3; ++q) {
      if (src[q])
        CK(cudaMemcpyAsync(stage, src[q], sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
      adj_launch_f3_to_f4(src[q] ? stage : nullptr, dst[q], (int)n, st);
    }
  }
  CK(cudaMemsetAsync(A.gH, 0, sizeof(float4) * cap * n, st));
  CK(cudaMemsetAsync(A.gW, 0, sizeof(float4) * kWallSlots * n, st));
  CK(cudaMemsetAsync(A.th, 0, sizeof(float) * 5 * n, st));
  const EnsGeom g = geom(e);
  for (cudaEvent_t& ev : a->ev)
    if (!ev) CK(cudaEventCreate(&ev));
  for (float& m : a->ms_phase) m = 0.0f;
  for (int s = a->nseg - 1; s >= 0 && (s + 1) * a->K > first; --s) {
    const int len = std::min(a->K, a->nsteps - s * a->K);
    const int q0 = std::max(0, first - s * a->K);   // first step of the segment to reverse
    TapeSeg& sg = a->seg[s];
    CK(cudaEventRecord(a->ev[0], st));
    if (!sg.valid) {
      int rc = restore_checkpoint(a, a->ck[s]);
      if (rc) return rc;
    }
    CK(cudaEventRecord(a->ev[1], st));
    if (!sg.valid) {
      int rc = record_segment(a, s, 0, a->words, sg);
      if (rc) return rc;
      if (!sg.valid) return -2;                  // one segment does not fit the tape
      for (int r = 0; r < s; ++r) a->seg[r].valid = false;
    }
    CK(cudaEventRecord(a->ev[2], st));
    for (int q = len - 1; q >= q0; --q) {
      const int t = s * a->K + q;
      adj_launch_step(g, a->tape, t, (int)n, A, st);
      if (sg.rb[q]) {
        adj_launch_unsort(a->tape, t, (int)n, A, st);
      } else {
        std::swap(A.gx, A.ix);
        std::swap(A.gv, A.iv);
        std::swap(A.gw, A.iw);
        std::swap(A.gH, A.iH);
        std::swap(A.gW, A.iW);
      }
    }
    CK(cudaEventRecord(a->ev[3], st));
    CK(cudaEventSynchronize(a->ev[3]));
    float m = 0.0f;
    for (int q = 0; q < 3; ++q) {
      CK(cudaEventElapsedTime(&m, a->ev[q], a->ev[q + 1]));
      a->ms_phase[q] += m;
    }
  }
  CK(cudaGetLastError());
  float* outs[3] = {gpos0, gvel0, gavel0};
  float4* srcs[3] = {A.gx, A.gv, A.gw};
  float* stage = reinterpret_cast<float*>(A.Fb);
  for (int q = 0; q < 3; ++q) {
    if (!outs[q]) continue;
    adj_launch_f4_to_f3(srcs[q], stage, (int)n, st);
    CK(cudaMemcpyAsync(outs[q], stage, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st));
  }
  if (gconst) {
    // positions of system s are [off_s, off_s + n_s) in every order the run
    // takes (keys sort by system first)
    adj_launch_sum_constants(A.th, a->d_sys_off, e->nsys, a->d_gconst, st);
    CK(cudaMemcpyAsync(gconst, a->d_gconst, sizeof(double) * 5 * e->nsys, cudaMemcpyDeviceToHost,
                       st));
  }
  CK(cudaStreamSynchronize(st));
  return sync_status(e);
}

}  // namespace

int blaze_ens_adj_backward(blaze_ens_adj* a, const float* gpos, const float* gvel,
                           const float* gavel, float* gpos0, float* gvel0, float* gavel0,
                           double* gconst) {
  return backward_impl(a, 0, gpos, gvel, gavel, gpos0, gvel0, gavel0, gconst);
}

int blaze_ens_adj_backward_window(blaze_ens_adj* a, int window, const float* gpos,
                                  const float* gvel, const float* gavel, float* gpos_w,
                                  float* gvel_w, float* gavel_w, double* gconst) {
  if (!a || window < 1 || window > a->nsteps) return -1;
  return backward_impl(a, a->nsteps - window, gpos, gvel, gavel, gpos_w, gvel_w, gavel_w,
                       gconst);
}

int blaze_ens_adj_profile(blaze_ens_adj* a, float* ms_restore, float* ms_record,
                          float* ms_reverse) {
  if (!a) return -1;
  if (ms_restore) *ms_restore = a->ms_phase[0];
  if (ms_record) *ms_record = a->ms_phase[1];
  if (ms_reverse) *ms_reverse = a->ms_phase[2];
  return 0;
}

int blaze_ens_adj_tape_info(blaze_ens_adj* a, unsigned long long* arena_bytes, int* on_tape,
                            unsigned long long* pool_bytes_max) {
  if (!a) return -1;
  if (arena_bytes) *arena_bytes = 4 * a->words;
  if (on_tape) *on_tape = a->on_tape;
  if (pool_bytes_max) *pool_bytes_max = 4 * a->pool_max;
  return 0;
}

int blaze_ens_adj_destroy(blaze_ens_adj* a) {
  if (!a) return -1;
  cudaStreamSynchronize(a->e->stream);
  free_adj(a);
  return 0;
}

}  // extern "C"
