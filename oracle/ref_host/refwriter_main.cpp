/*
 * The reference's state writer, Output_SystemState (V_02_2015/src/Input/
 * FileIO.h:12-315), run unmodified on a given state.  TEST INFRASTRUCTURE
 * ONLY: the CPU tests compare the library's writer with it byte for byte.
 *
 * FileIO.h reads the globals main.h defines (included unmodified from the
 * reference tree); this driver fills them from an input file, provides the
 * few host functions FileIO.h's other routines name (drawing and the
 * rotate-to-angle helpers, never called here), and answers the writer's
 * IDevice_Get_System_State with the loaded arrays.
 *
 * usage: refwriter INPUT RUN_DIR
 *   writes RUN_DIR/../Results/P/W/SystemState<time>.dat (Otype user)
 * INPUT (little-endian): int32 n, detail, sim_type, rotating_wobj,
 *   particle_type, revflag, rev_number, num_rem, rot_steps, steps_per_rev,
 *   n_p; float64 time, rot_angle; float32 energy[5], hatch_height, dt;
 *   float32 pos[3n], quat[4n], vel[3n], avel[3n], acc[3n]; uint32 type[n];
 *   int32 pid[n]; POBJ[n_p].
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>
using namespace std;

#include "main.h"

float Vel_Mill = 0.0f;
void Draw_DynamicGeometry() {}
void Rotate_VolObject_angle(float3) {}
void Rotate_WObject_angle(float3) {}

#include "Input/FileIO.h"

namespace {
std::vector<float3> g_pos, g_vel, g_avel, g_acc;
std::vector<Quaterion> g_q;
std::vector<uint> g_type;
std::vector<int> g_pid;
}  // namespace

void Device_Get_System_State(float3* pos, Quaterion* q, float3* vel, float3* avel, float3* acc,
                             uint* type, int* pid) {
  const size_t n = g_pos.size();
  if (pos) std::memcpy(pos, g_pos.data(), sizeof(float3) * n);
  if (q) std::memcpy(q, g_q.data(), sizeof(Quaterion) * n);
  if (vel) std::memcpy(vel, g_vel.data(), sizeof(float3) * n);
  if (avel) std::memcpy(avel, g_avel.data(), sizeof(float3) * n);
  if (acc) std::memcpy(acc, g_acc.data(), sizeof(float3) * n);
  if (type) std::memcpy(type, g_type.data(), sizeof(uint) * n);
  if (pid) std::memcpy(pid, g_pid.data(), sizeof(int) * n);
}

// named by FileIO.h's other routines (reading state files, surface forces);
// never called by the writer
void Device_Get_W_Forces(float3*, float3*) {}
void Device_Update_WorldObjectPostions(WOBJ*) {}
void Device_Update_DObjectPostions(DOBJ*) {}
void Device_Set_System_State(float3*, Quaterion*, float3*, float3*, float3*, uint*, int*) {}
void Device_Set_Tallys(float*) {}
void Device_Set_Pos(float3*, Quaterion*, uint*, int*) {}
void Device_Set_Pos_Velocity(float3*, Quaterion*, float3*, float3*, uint*, int*) {}

template <class T>
static bool rd(FILE* f, T* p, size_t count) { return fread(p, sizeof(T), count, f) == count; }

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  int h[11];
  double d[2];
  float fl[7];
  if (!rd(f, h, 11) || !rd(f, d, 2) || !rd(f, fl, 7)) return 4;
  const int n = h[0], n_p = h[10];
  g_pos.resize(n); g_q.resize(n); g_vel.resize(n); g_avel.resize(n); g_acc.resize(n);
  g_type.resize(n); g_pid.resize(n);
  if (!rd(f, g_pos.data(), n) || !rd(f, g_q.data(), n) || !rd(f, g_vel.data(), n) ||
      !rd(f, g_avel.data(), n) || !rd(f, g_acc.data(), n) || !rd(f, g_type.data(), n) ||
      !rd(f, g_pid.data(), n))
    return 5;
  std::vector<POBJ> pobj(std::max(n_p, 1));
  if (n_p > 0 && !rd(f, pobj.data(), n_p)) return 6;
  fclose(f);

  SimInfo.Num_Particles = n;
  SimInfo.particle_type = h[4];
  SimInfo.Rotating_WObject = h[3] != 0;
  SimInfo.InitalDelta_t = fl[6];
  m_sim_particle_type = h[4];
  m_Sim_Type = h[2];
  Revoution_number = h[6];
  m_Silo_SimData.flow_rate = h[7];
  m_Silo_SimData.hatch_height = fl[5];
  num_WrotSeps = h[8];
  m_Mill_SimData.Num_Steps_PerRev = h[9];
  simtime_elapsed = d[0];
  Rotation_Angle = d[1];
  for (int k = 0; k < 5; ++k) energy[k] = fl[k];
  m_KParticleObject = pobj.data();
  m_d_Particle_Pos = new float3[n];
  m_d_Particle_Quart = new Quaterion[n];
  m_d_Particle_Vel = new float3[n];
  m_d_Particle_RVel = new float3[n];
  m_d_Particle_Acc = new float3[n];
  m_d_Particle_Type = new uint[n];
  m_d_P_ID = new int[n];
  // the writer reads only get_InitPosGrid().grid_type (0: not a fill start)
  // and calls the non-virtual inline IDevice_Get_System_State
  static unsigned char ksd[sizeof(KSimulationData)];
  static unsigned char kdv[sizeof(KDevice)];
  std::memset(ksd, 0, sizeof(ksd));
  m_KSimulationData = reinterpret_cast<KSimulationData*>(ksd);
  m_KDevice = reinterpret_cast<KDevice*>(kdv);
  ProjectFolder = "P";
  WorldName = "W";
  if (chdir(argv[2]) != 0) return 7;
  mkdir("../Results", 0755);
  mkdir("../Results/P", 0755);
  mkdir("../Results/P/W", 0755);
  Output_SystemState(user, h[5], h[1]);
  return 0;
}
