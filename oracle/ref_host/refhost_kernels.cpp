/*
 * Oracle A: the reference's own DEM kernels, compiled as host C++ and driven
 * in the stage order of Device_DEM_UpdateSim (V_02_2015/src/Device/
 * DeviceInterface.cu:1825-2513, non-symmetric path, symplectic Euler,
 * Integration_Type 0).  TEST INFRASTRUCTURE ONLY: used by the parity tests,
 * the golden-fixture generator and bench.py's CPU-baseline leg; it is never
 * part of the product.
 *
 * The reference sources are #included unmodified from the reference tree
 * (the include path is given by oracle/Makefile); this file only provides
 * the device arrays that DeviceInterface.cu owns (DeviceInterface.cu:52-112),
 * a CPU "launch" helper, and a C entry point per stage so tests can read the
 * intermediate arrays (pair lists, forces) the reference keeps on the device.
 */
#include "prelude.h"

#include <algorithm>
#include <thrust/device_ptr.h>
#include <thrust/sort.h>
#include <vector>
#include <omp.h>

#include "DataStructures/KSimulationObjects.h"
#include "Utilities/Device/Opertators.cuh"
#include "Utilities/Device/Functions.cuh"
#include "Device/GPU_Memory_Transfer.cuh"
#include "Device/Utilities.cuh"
#include "Device/Computing/Collision_Detection_BroadPhase.cuh"
#include "Device/Computing/DEM_Kernels_Compute.cuh"

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

namespace {

/* Device arrays of DeviceInterface.cu:52-112, host-resident here. */
struct RefState {
  int n_max = 0, n_cur = 0, num_dead = 0, stepc = 0;
  int n_w = 0, n_p = 0, n_d = 0;
  bool cylinder_rotation = false;
  int threads = 1;
  std::vector<float3> pos, vel, acc, avel, f_pp, f_pp_ang, f_w, f_w_ang, f_l, f_l_ang;
  std::vector<Quaterion> ornt;
  std::vector<uint> ptype;
  std::vector<int> pid;
  std::vector<Contact_Info> lift_hist;
  std::vector<uint> hash;
  std::vector<int> hidx;
  std::vector<uint> cell_start, cell_end;
  std::vector<uint> nlist, nn;
  /* snapshot of the force arrays taken right before integration */
  bool capture = false;
  std::vector<float3> c_f_pp, c_f_pp_ang, c_f_w, c_f_w_ang, c_f_l, c_f_l_ang;
  int overflow = 0;
  double call_time = 0.0;
  /* the mill driver's lifter turn before every step (refh_set_dobj_rotation) */
  bool dobj_rot = false;
  float rot_ax = 0.0f, rot_ay = 0.0f, rot_rad = 0.0f;
  bool wobj_rot = false;
  float wrot_ax = 0.0f, wrot_ay = 0.0f, wrot_rad = 0.0f;
  int dobj_tr = -1;
  /* the mill's fill waves (refh_set_fill) */
  bool filling = false;
  int fill_pack = 0, fill_clear = 0, fill_counter = 0;
} S;

/* A volume object's faces from its vertices (Processing_Mills.h:27-58). */
void dobj_faces(DOBJ& D) {
  for (int j = 0; j < D.num_faces; ++j) {
    Surface& F = D.faces[j];
    float3 sum = make_float3(0.0f, 0.0f, 0.0f);
    for (int f = 0; f < F.num_vertex; ++f) sum = sum + D.vertex[F.vertex_Order[f]];
    F.centroid = (1.0f / F.num_vertex) * sum;
    const float3 v1 = D.vertex[F.vertex_Order[1]] - D.vertex[F.vertex_Order[0]];
    const float3 v2 = D.vertex[F.vertex_Order[2]] - D.vertex[F.vertex_Order[1]];
    const float3 v3 = D.vertex[F.vertex_Order[3]] - D.vertex[F.vertex_Order[2]];
    const float3 v4 = D.vertex[F.vertex_Order[0]] - D.vertex[F.vertex_Order[3]];
    const float3 n = cross(v2, v1);
    F.normal = n / length(n);
    F.area = 0.500000f * length(n) + 0.500000f * length(cross(v3, v4));
  }
}

/* Rotate_WObject_inc (Processing_Mills.h:257-334), restated on the
 * WorldObject array: the rotating objects' vertices turn by wrot_rad about
 * (wrot_ax, wrot_ay, 0), then every surface's centroid, normal and area. */
void rotate_wobj_inc() {
  const float c = std::cos(S.wrot_rad), sn = std::sin(S.wrot_rad);
  const float3 about = make_float3(S.wrot_ax, S.wrot_ay, 0.0f);
  for (int k = 0; k < Num_WorldObjects; ++k) {
    WOBJ& W = WorldObject[k];
    if (!W.is_rotating) continue;
    for (int v = 0; v < W.num_vertex; ++v) {
      const float3 p = W.vertex[v] - about;
      W.vertex[v].x = c * p.x + sn * p.y;
      W.vertex[v].y = -sn * p.x + c * p.y;
      W.vertex[v] = W.vertex[v] + about;
    }
    for (int j = 0; j < W.num_surfaces; ++j) {
      Surface& F = W.surfaces[j];
      float3 sum = make_float3(0.0f, 0.0f, 0.0f);
      for (int f = 0; f < F.num_vertex; ++f) sum = sum + W.vertex[F.vertex_Order[f]];
      F.centroid = (1.0f / F.num_vertex) * sum;
      const float3 v1 = W.vertex[F.vertex_Order[1]] - W.vertex[F.vertex_Order[0]];
      const float3 v2 = W.vertex[F.vertex_Order[2]] - W.vertex[F.vertex_Order[1]];
      const float3 n = cross(v2, v1);
      F.normal = n / length(n);
      if (F.num_vertex > 3) {
        const float3 v3 = W.vertex[F.vertex_Order[3]] - W.vertex[F.vertex_Order[2]];
        const float3 v4 = W.vertex[F.vertex_Order[0]] - W.vertex[F.vertex_Order[3]];
        F.area = 0.500000f * length(n) + 0.500000f * length(cross(v3, v4));
      } else {
        F.area = 0.500000f * length(n);
      }
    }
  }
}

/* Translate_VolObject (Processing_Mills.h:336-396), restated: object k moves
 * by its velocity times dt (main.cpp:176-180). */
void translate_dobj(int k) {
  DOBJ& D = DynamicObject[k];
  const float3 disp = D.velocity * SimParms.InitalDelta_t;
  for (int v = 0; v < D.num_vertex; ++v) D.vertex[v] += disp;
  dobj_faces(D);
  D.COM = D.COM + disp;
}

/* FP64 sums of the values the kernels add to the three energy tallies, in
 * the same order as the FP32 tallies (one host thread) or any order. */
double g_tally64[3] = {0.0, 0.0, 0.0};

/* Rotate_VolObject_Inc (Processing_Mills.h:4-75), restated on the uploaded
 * DynamicObject array (which Device_Update_DObjectPostions fills with the
 * host's turned copy, DeviceInterface.cu:2826-2831): the attached objects'
 * vertices and centre of mass turn by rot_rad about (rot_ax, rot_ay, 0),
 * then every face's centroid, normal and area follow from the vertices.
 * Single precision throughout, cos / sin of the float angle. */
void rotate_dobj_inc() {
  const float c = std::cos(S.rot_rad), sn = std::sin(S.rot_rad);
  const float3 about = make_float3(S.rot_ax, S.rot_ay, 0.0f);
  for (int k = 0; k < Num_DynamicObjects; ++k) {
    DOBJ& D = DynamicObject[k];
    if (!D.is_attached_DWorld) continue;
    for (int v = 0; v < D.num_vertex; ++v) {
      const float3 p = D.vertex[v] - about;
      D.vertex[v].x = c * p.x + sn * p.y;
      D.vertex[v].y = -sn * p.x + c * p.y;
      D.vertex[v] = D.vertex[v] + about;
    }
    for (int j = 0; j < D.num_faces; ++j) {
      Surface& F = D.faces[j];
      float3 sum = make_float3(0.0f, 0.0f, 0.0f);
      for (int f = 0; f < F.num_vertex; ++f) sum = sum + D.vertex[F.vertex_Order[f]];
      F.centroid = (1.0f / F.num_vertex) * sum;
      const float3 v1 = D.vertex[F.vertex_Order[1]] - D.vertex[F.vertex_Order[0]];
      const float3 v2 = D.vertex[F.vertex_Order[2]] - D.vertex[F.vertex_Order[1]];
      const float3 v3 = D.vertex[F.vertex_Order[3]] - D.vertex[F.vertex_Order[2]];
      const float3 v4 = D.vertex[F.vertex_Order[0]] - D.vertex[F.vertex_Order[3]];
      const float3 n = cross(v2, v1);
      F.normal = n / length(n);
      F.area = 0.500000f * length(n) + 0.500000f * length(cross(v3, v4));
    }
    const float3 p = D.COM - about;
    D.COM.x = c * p.x + sn * p.y;
    D.COM.y = -sn * p.x + c * p.y;
    D.COM = D.COM + about;
  }
}

/* Run `body` once per (block, thread) of a 1-D launch over n items. */
template <class F>
void launch(int n, F&& body) {
  const int B = 128;
  const int G = (n + B - 1) / B;
  if (G <= 0) return;
#pragma omp parallel for schedule(static) num_threads(S.threads)
  for (int b = 0; b < G; ++b) {
    blockIdx = make_uint3(b, 0, 0);
    blockDim = dim3(B, 1, 1);
    gridDim = dim3(G, 1, 1);
    for (int t = 0; t < B; ++t) {
      threadIdx = make_uint3(t, 0, 0);
      body();
    }
  }
}

}  // namespace

void refh_float_added(float* a, float v) {
  int k = -1;
  if (a == &Tally_EnergyDis_PP) k = 0;
  else if (a == &Tally_EnergyDisLift) k = 1;
  else if (a == &Tally_EnergyDisSurf) k = 2;
  if (k < 0) return;
#pragma omp atomic
  g_tally64[k] += (double)v;
}

extern "C" {

/* Mirrors Device_Set_SimulationData (DeviceInterface.cu:1499-1816) for a run
 * whose initial state is then set from a file: constants copied by value,
 * arrays sized to Num_Particles, forces and velocities zeroed
 * (Set_Init_Config_Device, GPU_Memory_Transfer.cuh:214-271). */
int refh_init(const SimulationInfo* si, const WOBJ* w, int n_w, const POBJ* p,
              int n_p, const DOBJ* d, int n_d) {
  if (!si || n_w < 0 || n_w > 8 || n_p < 1 || n_p > 8 || n_d < 0 || n_d > 32)
    return 1;
  S = RefState();
  SimParms = *si;
  std::memset(WorldObject, 0, sizeof(WorldObject));
  std::memset(ParticleObject, 0, sizeof(ParticleObject));
  std::memset(DynamicObject, 0, sizeof(DynamicObject));
  if (n_w) std::memcpy(WorldObject, w, sizeof(WOBJ) * n_w);
  std::memcpy(ParticleObject, p, sizeof(POBJ) * n_p);
  if (n_d) std::memcpy(DynamicObject, d, sizeof(DOBJ) * n_d);
  InitVel[0] = make_float3(0.0f, 0.0f, 0.0f);
  InitVel[1] = make_float3(0.0f, 0.0f, 0.0f);
  Num_WorldObjects = si->Num_WorldObjects;
  Num_ParticleObjects = si->Num_ParticleObjects;
  Num_DynamicObjects = n_d;
  Tally_EnergyDis_PP = Tally_EnergyDisLift = Tally_EnergyDisSurf = 0.0f;
  Tally_EnergyDis_Norm = Tally_EnergyDis_Shear = 0.0f;
  for (double& t : g_tally64) t = 0.0;
  Kill_count = 0;
  S.n_w = n_w; S.n_p = n_p; S.n_d = n_d;
  const int n = si->Num_Particles;
  S.n_max = S.n_cur = n;
  const float3 z = make_float3(0.0f, 0.0f, 0.0f);
  for (auto* v : {&S.pos, &S.vel, &S.acc, &S.avel, &S.f_pp, &S.f_pp_ang, &S.f_w,
                  &S.f_w_ang, &S.f_l, &S.f_l_ang})
    v->assign(n, z);
  Quaterion qi = {1.0f, 0.0f, 0.0f, 0.0f};
  S.ornt.assign(n, qi);
  S.ptype.assign(n, 0);
  S.pid.assign(n, 0);
  Contact_Info ci = {0, 0, 0, -1};
  S.lift_hist.assign(n, ci);
  S.hash.assign(n, 0);
  S.hidx.assign(n, 0);
  const int ncell = si->num_NNCells.x * si->num_NNCells.y * si->num_NNCells.z;
  S.cell_start.assign(ncell, 0xffffffffu);
  S.cell_end.assign(ncell, 0xffffffffu);
  /* Broad_List is N*32 in the reference (DeviceInterface.cu:2133); a little
   * slack keeps a >32 overflow from corrupting the host heap here. */
  S.nlist.assign(size_t(n + 64) * 32, 0);
  S.nn.assign(n, 0);
  return 0;
}

void refh_set_threads(int t) { S.threads = t < 1 ? 1 : t; }
void refh_set_capture(int on) { S.capture = on != 0; }
void refh_set_cylinder_rotation(int on) { S.cylinder_rotation = on != 0; }

/* Set_PSystem_State (GPU_Memory_Transfer.cuh:377-418): SpecType 3/4 upload. */
int refh_set_state(const float* pos3, const float* quat4, const float* vel3,
                   const float* avel3, const unsigned* type, const int* pid) {
  const int n = S.n_max;
  for (int i = 0; i < n; ++i) {
    S.pos[i] = make_float3(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]);
    if (SimParms.particle_type == 1 && quat4) {
      Quaterion q = {quat4[4 * i], quat4[4 * i + 1], quat4[4 * i + 2], quat4[4 * i + 3]};
      S.ornt[i] = q;
    }
    if (SimParms.sphere_orient) {
      Quaterion q = {1.0f, 0.0f, 0.0f, 0.0f};
      S.ornt[i] = q;
    }
    S.vel[i] = vel3 ? make_float3(vel3[3 * i], vel3[3 * i + 1], vel3[3 * i + 2])
                    : make_float3(0.0f, 0.0f, 0.0f);
    S.avel[i] = avel3 ? make_float3(avel3[3 * i], avel3[3 * i + 1], avel3[3 * i + 2])
                      : make_float3(0.0f, 0.0f, 0.0f);
    S.ptype[i] = type[i];
    S.pid[i] = pid[i];
  }
  return 0;
}

/* One call of Device_DEM_UpdateSim (DeviceInterface.cu:1825-2513). */
static int step_once() {
  const int n = S.n_cur;
  float3* P = S.pos.data();
  Quaterion* Q = S.ornt.data();
  float3* V = S.vel.data();
  float3* A = S.acc.data();
  float3* W = S.avel.data();
  uint* T = S.ptype.data();
  int* I = S.pid.data();
  Contact_Info* LH = S.lift_hist.data();

  /* 1. hash (DeviceInterface.cu:1884) */
  launch(n, [&] { Kernel_SpatialDecomp_CalcPHash(S.hash.data(), S.hidx.data(), P, n); });
  /* 2. stable sort (DeviceInterface.cu:1905 -> BroadPhase.cuh:110-117) */
  SpatialDecomp_ThrustSort_ByHash(S.hash.data(), S.hidx.data(), n);
  /* 3./4. gather into temporaries and copy back (DeviceInterface.cu:1960-2030) */
  {
    std::vector<float3> sp(n), sv(n), sa(n), sw(n), spo(1);
    std::vector<Quaterion> sq(n);
    std::vector<uint> st(n);
    std::vector<int> si(n);
    std::vector<Contact_Info> sl(n);
    launch(n, [&] {
      Kernel_SortArrays(S.hidx.data(), sp.data(), sq.data(), sv.data(), sw.data(), sa.data(),
                        st.data(), si.data(), sl.data(), nullptr, nullptr, spo.data(), P, Q,
                        V, W, A, T, I, LH, nullptr, nullptr, nullptr, n);
    });
    launch(n, [&] {
      Kernel_SpatialDecomp_ReorderPDA(sp.data(), sq.data(), sv.data(), sw.data(), sa.data(),
                                      st.data(), si.data(), sl.data(), nullptr, nullptr,
                                      spo.data(), P, Q, V, W, A, T, I, LH, nullptr, nullptr,
                                      nullptr, n);
    });
  }
  /* 5. drop killed particles (DeviceInterface.cu:2062-2091) */
  if (S.num_dead > 0) {
    S.n_cur -= S.num_dead;
    S.num_dead = 0;
    SimParms.Num_Particles = S.n_cur;
  }
  const int m = S.n_cur;
  /* 6. cell table (DeviceInterface.cu:2097-2105) */
  std::fill(S.cell_start.begin(), S.cell_start.end(), 0xffffffffu);
  std::fill(S.cell_end.begin(), S.cell_end.end(), 0xffffffffu);
  launch(m, [&] {
    Kernel_SpatialDecomp_BinData(S.hash.data(), S.cell_start.data(), S.cell_end.data(), m);
  });
  /* 7. contact list (DeviceInterface.cu:2146) */
  std::fill(S.nn.begin(), S.nn.end(), 0u);
  launch(m, [&] {
    Kernel_BroadCollisionDetection_NonSymmetry(S.cell_start.data(), S.cell_end.data(),
                                               S.nlist.data(), S.nn.data(), P, T, I, m);
  });
  for (int i = 0; i < m; ++i)
    if (S.nn[i] > 32) S.overflow = 1;
  /* 8. particle-particle forces (DeviceInterface.cu:2167/2204) */
  if (SimParms.particle_type == 0) {
    launch(m, [&] {
      Kernel_ParticleInteraction_Spheres_NonSymmetry(S.nn.data(), S.nlist.data(), P, V, W, T, I,
                                                     S.f_pp.data(), S.f_pp_ang.data(), m);
    });
  } else {
    launch(m, [&] {
      Kernel_ParticleInteraction_Polyhedra_NonSymmetry(S.nn.data(), S.nlist.data(), P, Q, V, W,
                                                       A, T, I, S.f_pp.data(),
                                                       S.f_pp_ang.data(), m);
    });
  }
  /* 9. volume objects / lifters (DeviceInterface.cu:2316-2329) */
  if (S.n_d > 0) {
    launch(m, [&] {
      VolumeObject_InteractionParticle(S.f_l.data(), S.f_l_ang.data(), LH, P, Q, V, W, A, T, I,
                                       m);
    });
  }
  /* 10. world objects (DeviceInterface.cu:2342) */
  launch(m, [&] {
    WorldObject_InteractionParticle(false, S.cylinder_rotation, S.f_w.data(), S.f_w_ang.data(),
                                    nullptr, P, Q, V, W, A, T, I, m);
  });
  if (S.capture) {
    S.c_f_pp = S.f_pp; S.c_f_pp_ang = S.f_pp_ang;
    S.c_f_w = S.f_w; S.c_f_w_ang = S.f_w_ang;
    S.c_f_l = S.f_l; S.c_f_l_ang = S.f_l_ang;
  }
  /* 11. integrate (DeviceInterface.cu:2394) */
  launch(m, [&] {
    Integrate_Euler_NonSymmetry(S.f_pp.data(), S.f_pp_ang.data(), S.f_w.data(), S.f_w_ang.data(),
                                S.f_l.data(), S.f_l_ang.data(), P, Q, V, W, T, I, m);
  });
  /* 13. silo kill check every 1000 steps (DeviceInterface.cu:2463-2498) */
  if (SimParms.Kill_Particles) {
    S.stepc++;
    if (S.stepc >= 1000) {
      if (SimParms.Rotating_WObject)
        launch(m, [&] { Remove_PL_Discharged_Particles(P, I, m); });
      else
        launch(m, [&] { Remove_Silo_Discharged_Particles(P, I, m); });
      int killed[2];
      blockIdx = make_uint3(0, 0, 0);
      threadIdx = make_uint3(0, 0, 0);
      Kill_copy(killed);
      S.num_dead = killed[0];
      S.stepc = 0;
    }
  }
  S.call_time += SimParms.InitalDelta_t;
  return 0;
}

int refh_step(int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    /* Device_DEM_UpdateSim's wave control and Fill_State
       (DeviceInterface.cu:1055-1110, 1840-1866), restated */
    if (S.filling) {
      if (S.fill_counter > S.fill_clear || S.n_cur == 0) {
        S.fill_counter = 0;
        if (S.n_cur < S.n_max) {
          S.n_cur += std::min(S.fill_pack, S.n_max - S.n_cur);
          SimParms.Num_Particles = S.n_cur;
        }
        if (S.n_cur >= S.n_max) S.filling = false;
      } else {
        S.fill_counter++;
      }
    }
    if (S.wobj_rot) rotate_wobj_inc();
    if (S.dobj_rot) rotate_dobj_inc();
    if (S.dobj_tr >= 0) translate_dobj(S.dobj_tr);
    int rc = step_once();
    if (rc) return rc;
  }
  return S.overflow ? 2 : 0;
}

int refh_num_current(void) { return S.n_cur; }

/* Get_SystemState (GPU_Memory_Transfer.cuh:486-520): current memory order. */
int refh_get_state(float* pos3, float* quat4, float* vel3, float* avel3, unsigned* type,
                   int* pid) {
  const int n = S.n_max;
  for (int i = 0; i < n; ++i) {
    float3 p = S.pos[i];
    if (SimParms.particle_type != 0) p = p - ParticleObject[S.ptype[i]].COM;
    if (pos3) { pos3[3 * i] = p.x; pos3[3 * i + 1] = p.y; pos3[3 * i + 2] = p.z; }
    if (quat4) {
      quat4[4 * i] = S.ornt[i].w; quat4[4 * i + 1] = S.ornt[i].x;
      quat4[4 * i + 2] = S.ornt[i].y; quat4[4 * i + 3] = S.ornt[i].z;
    }
    if (vel3) { vel3[3 * i] = S.vel[i].x; vel3[3 * i + 1] = S.vel[i].y; vel3[3 * i + 2] = S.vel[i].z; }
    if (avel3) { avel3[3 * i] = S.avel[i].x; avel3[3 * i + 1] = S.avel[i].y; avel3[3 * i + 2] = S.avel[i].z; }
    if (type) type[i] = S.ptype[i];
    if (pid) pid[i] = S.pid[i];
  }
  return 0;
}

static void put3(float* dst, const std::vector<float3>& v) {
  if (!dst) return;
  for (size_t i = 0; i < v.size(); ++i) {
    dst[3 * i] = v[i].x; dst[3 * i + 1] = v[i].y; dst[3 * i + 2] = v[i].z;
  }
}

/* Force arrays of the last step as they stood before integration. */
int refh_get_forces(float* f_pp, float* f_pp_ang, float* f_w, float* f_w_ang, float* f_l,
                    float* f_l_ang) {
  if (!S.capture || S.c_f_pp.empty()) return 1;
  put3(f_pp, S.c_f_pp); put3(f_pp_ang, S.c_f_pp_ang);
  put3(f_w, S.c_f_w); put3(f_w_ang, S.c_f_w_ang);
  put3(f_l, S.c_f_l); put3(f_l_ang, S.c_f_l_ang);
  return 0;
}

/* Contact list of the last step: NN_NUM[i] and Broad_List[i*32+k]. */
int refh_get_nlist(unsigned* nn, unsigned* list) {
  const int n = S.n_cur;
  for (int i = 0; i < n; ++i) {
    nn[i] = S.nn[i];
    for (int k = 0; k < 32; ++k) list[32 * i + k] = k < (int)S.nn[i] ? S.nlist[32 * i + k] : 0u;
  }
  return 0;
}

/* Cell table of the last step. */
int refh_get_cells(unsigned* start, unsigned* end) {
  std::copy(S.cell_start.begin(), S.cell_start.end(), start);
  std::copy(S.cell_end.begin(), S.cell_end.end(), end);
  return 0;
}

/* Lifter contact history (cont_type per particle) of the last step. */
int refh_get_lifter_hist(int* cont_type) {
  for (int i = 0; i < S.n_max; ++i) cont_type[i] = S.lift_hist[i].cont_type;
  return 0;
}

/* GetEnergy (GPU_Memory_Transfer.cuh:604-619) with NumPhysicsTallies = 3. */
int refh_get_energy(float* e3) {
  e3[0] = Tally_EnergyDis_PP * 1E-4;
  e3[1] = Tally_EnergyDisLift * 1E-4;
  e3[2] = Tally_EnergyDisSurf * 1E-4;
  return 0;
}

int refh_update_wobj(const WOBJ* w, int n_w) {
  if (n_w < 0 || n_w > 8) return 1;
  std::memcpy(WorldObject, w, sizeof(WOBJ) * n_w);
  return 0;
}

void refh_set_dobj_rotation(float about_x, float about_y, float rad_per_step, int on) {
  S.dobj_rot = on != 0;
  S.rot_ax = about_x;
  S.rot_ay = about_y;
  S.rot_rad = rad_per_step;
}

void refh_set_wobj_rotation(float about_x, float about_y, float rad_per_step, int on) {
  S.wobj_rot = on != 0;
  S.wrot_ax = about_x;
  S.wrot_ay = about_y;
  S.wrot_rad = rad_per_step;
}

void refh_set_dobj_translation(int index, int on) { S.dobj_tr = on ? index : -1; }

/* A fill run: nothing in the run until the first step's wave, then `pack`
 * particles (the next ones in memory order) every clear + 1 steps. */
void refh_set_fill(int pack, int clear) {
  S.filling = pack > 0;
  S.fill_pack = pack;
  S.fill_clear = clear;
  S.fill_counter = 0;
  S.n_cur = 0;
  SimParms.Num_Particles = 0;
}

int refh_get_wobj(WOBJ* w, int n_w) {
  if (n_w < 0 || n_w > 8) return 1;
  std::memcpy(w, WorldObject, sizeof(WOBJ) * n_w);
  return 0;
}

int refh_get_dobj(DOBJ* d, int n_d) {
  if (n_d < 0 || n_d > 32) return 1;
  std::memcpy(d, DynamicObject, sizeof(DOBJ) * n_d);
  return 0;
}

void refh_set_energy(const float* raw3) {
  Tally_EnergyDis_PP = raw3 ? raw3[0] : 0.0f;
  Tally_EnergyDisLift = raw3 ? raw3[1] : 0.0f;
  Tally_EnergyDisSurf = raw3 ? raw3[2] : 0.0f;
  for (int k = 0; k < 3; ++k) g_tally64[k] = raw3 ? (double)raw3[k] : 0.0;
}

/* The FP64 sums of the same values, in GetEnergy's units (x 1e-4). */
int refh_get_energy64(double* e3) {
  for (int k = 0; k < 3; ++k) e3[k] = g_tally64[k] * 1E-4;
  return 0;
}

int refh_update_dobj(const DOBJ* d, int n_d) {
  if (n_d < 0 || n_d > 32) return 1;
  std::memcpy(DynamicObject, d, sizeof(DOBJ) * n_d);
  return 0;
}

/* Device_OpenHatch (DeviceInterface.cu:2859-2869): re-upload, drop the last
 * world object. */
int refh_open_hatch(const WOBJ* w, int n_w) {
  int rc = refh_update_wobj(w, n_w);
  if (rc) return rc;
  Num_WorldObjects = Num_WorldObjects - 1;
  return 0;
}

/* Byte sizes of the boundary structs as the reference's own headers lay them
 * out, for the layout checks of the product's mirror header. */
int refh_sizeof(const char* name) {
  std::string s(name);
  if (s == "SimulationInfo") return sizeof(SimulationInfo);
  if (s == "POBJ") return sizeof(POBJ);
  if (s == "WOBJ") return sizeof(WOBJ);
  if (s == "DOBJ") return sizeof(DOBJ);
  if (s == "InitConfig") return sizeof(InitConfig);
  if (s == "Surface") return sizeof(Surface);
  if (s == "Macro_Cylinder") return sizeof(Macro_Cylinder);
  if (s == "PP_Parms") return sizeof(PP_Parms);
  if (s == "Quaterion") return sizeof(Quaterion);
  if (s == "Contact_Info") return sizeof(Contact_Info);
  return -1;
}

}  // extern "C"
