// A headless driver of the reference's own KDevice wrapper
// (Interface/KDevice.{h,cpp}, compiled unchanged against
// include/kdevice/Device/DeviceInterface.h) linked against libblaze_b200.so:
// the integration of INTEGRATION.md section 1, built and run by the tests.
// Test infrastructure: it reads one simulation's boundary structs and state
// from a file, steps it through KDevice and writes the state back.
//
//   kdevice_headless IN OUT STEPS
//
// IN:  int32 [magic, N, n_w, n_p, n_d, cylinder rotation,
//             sizeof SimulationInfo, WOBJ, POBJ, DOBJ], then SimulationInfo,
//      WOBJ[8], POBJ[8], DOBJ[32], and N x (pos float3), (vel float3),
//      (avel float3), type uint32, P_ID int32 (array by array)
// OUT: the state after STEPS calls of IDevice_DEM_UpdateSim, same arrays in
//      memory order; exit status = the library's status bits (0 = clean).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "KDevice.h"

namespace {

constexpr int kMagic = 0x4B444556;

bool rd(std::FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }
bool wr(std::FILE* f, const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s IN OUT STEPS\n", argv[0]);
    return 2;
  }
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int h[10];
  if (!rd(f, h, sizeof(h)) || h[0] != kMagic || h[6] != (int)sizeof(SimulationInfo) ||
      h[7] != (int)sizeof(WOBJ) || h[8] != (int)sizeof(POBJ) || h[9] != (int)sizeof(DOBJ)) {
    std::fprintf(stderr, "kdevice_headless: input layout does not match this build\n");
    return 2;
  }
  const int n = h[1], n_w = h[2], n_p = h[3], n_d = h[4], cyl_rot = h[5];
  SimulationInfo si;
  std::vector<WOBJ> w(8);
  std::vector<POBJ> p(8);
  std::vector<DOBJ> d(32);
  std::vector<float3> pos(n), vel(n), avel(n), acc(n);
  std::vector<uint> type(n);
  std::vector<int> pid(n);
  bool ok = rd(f, &si, sizeof(si)) && rd(f, w.data(), sizeof(WOBJ) * 8) &&
            rd(f, p.data(), sizeof(POBJ) * 8) && rd(f, d.data(), sizeof(DOBJ) * 32) &&
            rd(f, pos.data(), sizeof(float3) * n) && rd(f, vel.data(), sizeof(float3) * n) &&
            rd(f, avel.data(), sizeof(float3) * n) && rd(f, type.data(), sizeof(uint) * n) &&
            rd(f, pid.data(), sizeof(int) * n);
  std::fclose(f);
  if (!ok) return 2;
  si.Num_ParticlesPerObject = nullptr;   // a host pointer of the writer's process
  InitConfig ic;
  std::memset(&ic, 0, sizeof(ic));
  ic.use_file = true;                    // the state comes from the caller, as from a state file

  KDevice dev(w.data(), p.data(), d.data(), n_w, n_p, n_d, &si, &ic);
  if (cyl_rot) dev.IDevice_drum_rotation(true);
  dev.IDevice_Set_ParticleSystem_State(pos.data(), nullptr, vel.data(), avel.data(), nullptr,
                                       type.data(), pid.data());
  const int steps = std::atoi(argv[3]);
  for (int k = 0; k < steps; ++k) dev.IDevice_DEM_UpdateSim();
  dev.IDevice_Get_System_State(pos.data(), nullptr, vel.data(), avel.data(), acc.data(),
                               type.data(), pid.data());
  const int status = blaze_sync(blaze_default_sim());
  dev.clean();

  std::FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 2;
  ok = wr(o, pos.data(), sizeof(float3) * n) && wr(o, vel.data(), sizeof(float3) * n) &&
       wr(o, avel.data(), sizeof(float3) * n) && wr(o, type.data(), sizeof(uint) * n) &&
       wr(o, pid.data(), sizeof(int) * n);
  std::fclose(o);
  if (!ok) return 2;
  return status < 0 ? 3 : (status > 0 ? 4 : 0);
}
