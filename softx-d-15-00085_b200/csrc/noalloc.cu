// noalloc.cu -- blaze_contact_list_static: the broad phase of the step (cell
// keys, stable radix sort, cell table, contact list) for callers that cannot
// allocate device memory.
//
// Who needs it: a host code that calls the broad phase between its own
// kernels -- a coupled CFD-DEM or FEM solver, a renderer's particle pass --
// often may not allocate.  cudaMalloc and cudaFree synchronise the whole
// device and would stall that caller's pipeline, and many such hosts hand
// out all device memory from their own pool at start-up and forbid further
// allocation.  The handle API (blaze_create) allocates its buffers once; this
// entry point allocates nothing at all.
//
// Its working memory is one file-scope __device__ array (kScratchBytes,
// about 5.8 MB), which every GPU that loads the library holds until the
// process exits.  That bounds the problem size: at most kMaxParticles
// spheres and kMaxCells hash-table entries; larger calls are rejected.
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in), so the device address is looked up with
// cudaGetSymbolAddress once per device, on the first call made with that
// device current; make that first call before any stream capture.
//
// Every call shares the one array and leaves its contents behind; each call
// re-initialises what it relies on (control words, pid copy, cell table).
// Two calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on the array and corrupt each other's
// results: serialise them.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "blaze_dem.h"
#include "dem_kernels.cuh"
#include "radix_sort.cuh"

using namespace blaze;

namespace {

constexpr int kMaxParticles = 65536;
constexpr uint32_t kMaxCells = 262144;
constexpr int kMaxDevices = 64;
constexpr int kMaxTilesStatic = (kMaxParticles + kTileKeys - 1) / kTileKeys;

constexpr size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the pieces inside the scratch array.
constexpr size_t kOffParams = 0;
constexpr size_t kOffCtl = up256(kOffParams + sizeof(SimParams));
constexpr size_t kOffKeys0 = up256(kOffCtl + sizeof(StepCtl));
constexpr size_t kOffKeys1 = up256(kOffKeys0 + sizeof(uint32_t) * kMaxParticles);
constexpr size_t kOffVals0 = up256(kOffKeys1 + sizeof(uint32_t) * kMaxParticles);
constexpr size_t kOffVals1 = up256(kOffVals0 + sizeof(int32_t) * kMaxParticles);
constexpr size_t kOffCounts = up256(kOffVals1 + sizeof(int32_t) * kMaxParticles);
constexpr size_t kOffTotals = up256(kOffCounts + sizeof(uint32_t) * kRadixDigits * kMaxTilesStatic);
constexpr size_t kOffPid0 = up256(kOffTotals + sizeof(uint32_t) * kRadixDigits);
constexpr size_t kOffPid1 = up256(kOffPid0 + sizeof(int) * kMaxParticles);
constexpr size_t kOffSorted = up256(kOffPid1 + sizeof(int) * kMaxParticles);
constexpr size_t kOffSpare = up256(kOffSorted + sizeof(float4) * kMaxParticles);
constexpr size_t kOffCstart = up256(kOffSpare + sizeof(float4) * kMaxParticles);
constexpr size_t kOffCend = up256(kOffCstart + sizeof(uint32_t) * kMaxCells);
constexpr size_t kScratchBytes = up256(kOffCend + sizeof(uint32_t) * kMaxCells);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char* g_base[kMaxDevices] = {};

// What the broad-phase kernels read from SimParams, passed by value to the
// kernel that writes the call's parameters and control words into the
// scratch array (no copy from host memory).
struct StaticParams {
  float3 origin, cell;
  int3 ncells;
  uint32_t ncell_tab;
  float skin;
  int max_nbr;
  int n;
};

static_assert(sizeof(SimParams) % 4 == 0 && sizeof(StepCtl) % 4 == 0, "zeroed as 32-bit words");

// One block: zeroes the SimParams and StepCtl slots, then sets the fields
// the hash, reorder and contact-list kernels read.
__global__ void k_static_init(StaticParams sp, SimParams* dp, StepCtl* ctl) {
  uint32_t* pw = reinterpret_cast<uint32_t*>(dp);
  uint32_t* cw = reinterpret_cast<uint32_t*>(ctl);
  for (size_t k = threadIdx.x; k < sizeof(SimParams) / 4; k += blockDim.x) pw[k] = 0u;
  for (size_t k = threadIdx.x; k < sizeof(StepCtl) / 4; k += blockDim.x) cw[k] = 0u;
  __syncthreads();
  if (threadIdx.x != 0) return;
  dp->origin = sp.origin;
  dp->cell = sp.cell;
  dp->ncells = sp.ncells;
  dp->ncell_tab = sp.ncell_tab;
  dp->skin = sp.skin;
  dp->max_nbr = sp.max_nbr;
  ctl->n_cur = sp.n;
}

int cuda_fail(cudaError_t e) {
  std::fprintf(stderr, "blaze: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
  return -(1000 + (int)e);
}

// Device address of g_scratch on the current device (looked up once per
// device; host code must never pass g_scratch itself to a kernel).
int scratch_base(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e);
  if (dev < 0 || dev >= kMaxDevices) return -1;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_base[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return cuda_fail(e);
    g_base[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_base[dev];
  return 0;
}

}  // namespace

extern "C" int blaze_contact_list_static(const float* pos4, int n, const SimulationInfo* si,
                                         float skin, int max_nbr, int* perm, uint* nn,
                                         uint* list, uint* status, void* stream) {
  if (!pos4 || !si || !perm || !nn || !list || n < 1 || max_nbr < 1 || !(skin >= 0.0f))
    return -1;
  const long long nx = si->num_NNCells.x, ny = si->num_NNCells.y, nz = si->num_NNCells.z;
  if (nx < 1 || ny < 1 || nz < 1) return -1;
  // hash-table entries: the largest in-grid hash + 1 (the hash aliases when
  // nx != nz, as the reference's does), at least the cell count
  const long long hmax = (nx - 1) + (nz - 1) * nz + (ny - 1) * nx * nz + 1;
  const long long ntab = hmax > nx * ny * nz ? hmax : nx * ny * nz;
  if (n > kMaxParticles || ntab > (long long)kMaxCells) {
    std::fprintf(stderr,
                 "blaze_contact_list_static: %d particles / %lld hash cells exceed the built-in "
                 "scratch (at most %d particles and %u cells); use the handle API instead\n",
                 n, ntab, kMaxParticles, kMaxCells);
    return -3;
  }
  unsigned char* base = nullptr;
  int rc = scratch_base(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  StaticParams sp;
  sp.origin = si->worldOrigin;
  sp.cell = si->cellSize;
  sp.ncells = si->num_NNCells;
  sp.ncell_tab = (uint32_t)ntab;
  sp.skin = skin;
  sp.max_nbr = max_nbr;
  sp.n = n;

  SimParams* dp = reinterpret_cast<SimParams*>(base + kOffParams);
  StepCtl* ctl = reinterpret_cast<StepCtl*>(base + kOffCtl);
  RadixSortBuffers rs;
  rs.keys[0] = reinterpret_cast<uint32_t*>(base + kOffKeys0);
  rs.keys[1] = reinterpret_cast<uint32_t*>(base + kOffKeys1);
  rs.vals[0] = reinterpret_cast<int32_t*>(base + kOffVals0);
  rs.vals[1] = reinterpret_cast<int32_t*>(base + kOffVals1);
  rs.counts = reinterpret_cast<uint32_t*>(base + kOffCounts);
  rs.totals = reinterpret_cast<uint32_t*>(base + kOffTotals);
  rs.max_n = kMaxParticles;
  rs.max_tiles = kMaxTilesStatic;
  OrderBuf ob{};
  ob.pid[0] = reinterpret_cast<int*>(base + kOffPid0);
  ob.pid[1] = reinterpret_cast<int*>(base + kOffPid1);
  uint32_t* cstart = reinterpret_cast<uint32_t*>(base + kOffCstart);
  uint32_t* cend = reinterpret_cast<uint32_t*>(base + kOffCend);
  float4* in4 = const_cast<float4*>(reinterpret_cast<const float4*>(pos4));
  float4* sorted = reinterpret_cast<float4*>(base + kOffSorted);
  float4* spare = reinterpret_cast<float4*>(base + kOffSpare);
  // the reorder kernel also moves velocities; here they are not wanted, so
  // it reads the positions twice and writes both copies into one spare buffer
  const StateBuf src{in4, in4, in4};
  const StateBuf dst{sorted, spare, spare};

  int bits = 1;
  const uint32_t top = (uint32_t)ntab + 1u;
  while (bits < 32 && (top >> bits) != 0) bits++;

#define CKS(x)                                    \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_);  \
  } while (0)
  // what this call relies on starting from a known value
  k_static_init<<<1, 256, 0, st>>>(sp, dp, ctl);
  CKS(cudaMemsetAsync(ob.pid[0], 0, sizeof(int) * n, st));  // every particle live
  CKS(cudaMemsetAsync(cstart, 0xff, sizeof(uint32_t) * ntab, st));
  launch_hash(dp, src, ob, n, rs.keys[0], ctl, nullptr, st);
  const int res = radix_sort_pairs(rs, n, bits, true, nullptr, st);
  launch_reorder(src, dst, ob, n, rs.keys[res], rs.vals[res], cstart, cend, (uint32_t)ntab,
                 false, nullptr, ctl, nullptr, st);
  NbrList nl;
  nl.idx = list;
  nl.cnt = nn;
  nl.stride = n;
  nl.cap = max_nbr;
  nl.flat = nullptr;
  nl.flat_n = nullptr;
  launch_nlist(dp, dst, n, cstart, cend, nl, ctl, nullptr, st);
  CKS(cudaMemcpyAsync(perm, rs.vals[res], sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  if (status)
    CKS(cudaMemcpyAsync(status, &ctl->status, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  CKS(cudaGetLastError());
#undef CKS
  return 0;
}
