/*
 * blaze_dem.h -- C ABI of the B200 DEM step library (libblaze_b200.so).
 *
 * Part 1 mirrors the reference's simulation-step interface
 * (V_02_2015/src/Device/DeviceInterface.h:16-95) name for name, so the
 * reference's KDevice wrapper (V_02_2015/src/Interface/KDevice.h:17-99) and
 * its callers compile against this header unchanged.  Differences in the
 * contract, all deliberate:
 *   - C linkage and an int status instead of void + exit(1):
 *       0  ok
 *       >0 StatusBits raised by the kernels since the last call that
 *          synchronised (1 list overflow, 2 particle outside the grid,
 *          4 non-finite state, 8 particle type outside the table,
 *          16 bounded device wait gave up, 32 a polyhedron contact met a
 *          case the reference leaves undefined and got the library's
 *          defined result, 64 with a neighbour-list skin: a particle passed
 *          half the skin inside a block of steps with no list check, so
 *          contacts may have been missed, 128 with a skin: 2 r + skin of
 *          some sphere exceeds a cell edge of the grid the list is searched
 *          on (only blaze_contact_list_static can raise it: with a skin the
 *          handle API searches a grid of cells at least 2 r_max + skin over
 *          the project grid's extent))
 *       <0 -(1000 + cudaError_t) for a CUDA error, -1 bad argument,
 *          -2 no simulation set up
 *   - Device_DEM_UpdateSim only enqueues the step on the library's stream;
 *     every Get/Set call orders after it, so callers observe the reference's
 *     synchronous semantics.  Option sync_each_step=1 makes every step block.
 *   - Removed particles are counted per check (the reference's Kill_count is
 *     never reset, DeviceInterface.cu:2494).
 * One simulation per process through Part 1, as in the reference.
 *
 * Part 2 (blaze_*) is additive: handles for several independent
 * simulations, options (neighbour-list skin and capacity, wall culling,
 * CUDA-graph stepping), device-resident state access and parity hooks.
 */
#ifndef BLAZE_DEM_H_
#define BLAZE_DEM_H_

#include "blaze_types.h"

#ifndef __cplusplus
#include <stdbool.h> /* drum_rotation(bool) */
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- Part 1 */

/* DeviceInterface.h:16-20 / DeviceInterface.cu:1499 */
int Device_Set_SimulationData(WOBJ* h_WorldOBJ, POBJ* h_ParticleOBJ, DOBJ* h_DynamicOBJ,
                              SimulationInfo* h_SimInfo, int h_Num_WorldOBJ,
                              int h_Num_ParticleOBJ, int h_Num_DynamicOBJ,
                              InitConfig* h_PosConfig);
/* DeviceInterface.h:23-24 / DeviceInterface.cu:1116 (SpecType 1) */
int Device_Set_Pos(float3* h_pos, Quaterion* h_Ornt, uint* h_ptype, int* h_pid);
/* DeviceInterface.h:27-29 / DeviceInterface.cu:1209 (SpecType 2) */
int Device_Set_Pos_Velocity(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            uint* h_ptype, int* h_pid);
/* DeviceInterface.h:32-35 / DeviceInterface.cu:1307 (SpecType 3/4; h_acc ignored, as there) */
int Device_Set_System_State(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            float3* h_acc, uint* h_ptype, int* h_pid);
/* DeviceInterface.h:38 / DeviceInterface.cu:1429 */
int Device_Set_Tallys(float* h_Tallys);
/* DeviceInterface.h:44-49 / DeviceInterface.cu:2613 */
int Device_Get_System_State(float3* h_pos, Quaterion* h_Ornt, float3* h_vel, float3* h_Avel,
                            float3* h_acc, uint* h_ptype, int* h_pid);
/* DeviceInterface.h:52-53 / DeviceInterface.cu:2524 */
int Device_Get_P_Positions(float3* Pos, Quaterion* Quart_ornt, uint* h_ptype, int* h_pid);
/* DeviceInterface.h:56-57 / DeviceInterface.cu:2692 */
int Device_Get_P_Velocity(float3* H_Vel, float3* H_Rvel, int Flag, uint* h_ptype, int* h_pid);
/* DeviceInterface.h:63 / DeviceInterface.cu:2769: wall force of the last step */
int Device_Get_W_Forces(float3* WallForces, float3* WallContact_Point);
/* DeviceInterface.h:65 / DeviceInterface.cu:2795 */
int Device_Get_Energy(float* Energy);
/* DeviceInterface.h:74 / DeviceInterface.cu:2826 */
int Device_Update_DObjectPostions(DOBJ* h_DynamicOBJ);
/* DeviceInterface.h:75 / DeviceInterface.cu:2838 */
int Device_Update_WorldObjectPostions(WOBJ* h_WorldOBJ);
/* DeviceInterface.h:77 / DeviceInterface.cu:2859 */
int Device_OpenHatch(WOBJ* h_WorldOBJ, int h_Num_WorldOBJ);
/* DeviceInterface.h:78 / DeviceInterface.cu:2902 */
int Device_Clean(void);
/* DeviceInterface.h:79 / DeviceInterface.cu:2787 */
int Device_Reset_Energy(int num_values);
/* DeviceInterface.h:82 / DeviceInterface.cu:2848 */
int drum_rotation(bool cylinder_rotation);
/* DeviceInterface.h:83 / DeviceInterface.cu:2781 */
int Start_Bin(void);
/* DeviceInterface.h:85-87 / DeviceInterface.cu:2872-2893 */
int Device_AddForce(void);
int Device_SubForce(void);
int Device_ZeroForce(void);
/* DeviceInterface.h:95 / DeviceInterface.cu:1825 */
int Device_DEM_UpdateSim(void);

/* ---------------------------------------------------------------- Part 2 */

typedef struct blaze_sim blaze_sim;

typedef struct blaze_options {
  float skin;          /* neighbour-list skin, cm; 0 = contacts only, rebuilt every step */
  int max_nbr;         /* neighbour slots per particle (reference: 32) */
  int wall_grid;       /* 1 = cull wall faces per cell (exact), 0 = test every face */
  int use_graph;       /* 1 = step through a captured CUDA graph */
  int capture_forces;  /* 1 = keep the last step's per-particle forces (parity hooks) */
  int sync_each_step;  /* 1 = every step blocks and returns its status */
  int fast_law;        /* 1 = the sphere particle-particle law in contracted form
                        * (fused multiply-adds, approximate reciprocals): contact
                        * sets unchanged, forces within 1e-5 relative of the
                        * reference's arithmetic instead of bit for bit; steps
                        * with energy tallies keep the reference's arithmetic */
} blaze_options;

/* Library defaults: skin 0, max_nbr 32, wall_grid 1, use_graph 0,
 * capture_forces 0, sync_each_step 0, fast_law 0 (the reference's
 * semantics). */
void blaze_default_options(blaze_options* o);

int blaze_create(blaze_sim** out, const WOBJ* w, int n_w, const POBJ* p, int n_p, const DOBJ* d,
                 int n_d, const SimulationInfo* si, const blaze_options* opt);
int blaze_destroy(blaze_sim* s);
int blaze_set_options(blaze_sim* s, const blaze_options* opt);
int blaze_set_cylinder_rotation(blaze_sim* s, int on);
/* Host arrays, AoS float3 / int, length Num_Particles (vel/avel may be NULL). */
int blaze_set_state(blaze_sim* s, const float* pos3, const float* vel3, const float* avel3,
                    const uint* type, const int* pid);
int blaze_get_state(blaze_sim* s, float* pos3, float* vel3, float* avel3, uint* type, int* pid);
/* The same with orientations, (w, x, y, z) per particle (Quaterion order;
 * NULL = identity on set, not returned on get).  Polyhedra (particle_type
 * 1): positions are set as centres of mass and returned relative to the
 * object file's origin (pos - COM), as Set_PSystem_State / Get_SystemState
 * do (GPU_Memory_Transfer.cuh:400-440, 486-520). */
int blaze_set_state_ornt(blaze_sim* s, const float* pos3, const float* quat4, const float* vel3,
                         const float* avel3, const uint* type, const int* pid);
int blaze_get_state_ornt(blaze_sim* s, float* pos3, float* quat4, float* vel3, float* avel3,
                         uint* type, int* pid);
/* Enqueue nsteps steps (asynchronous unless sync_each_step; with
 * use_graph = 1 no step waits for the host: the list checks of a skin are
 * decided on the device).  With use_graph = 1 the graphs are built on first
 * use; blaze_prepare_graphs builds them ahead. */
int blaze_step(blaze_sim* s, int nsteps);
/* Instantiate every CUDA graph that graph stepping with the current options
 * launches (both buffer parities; with a skin the block graph and the
 * one-step graphs), so that no stream capture or instantiation happens
 * inside a later blaze_step.  Changing options or moves drops them. */
int blaze_prepare_graphs(blaze_sim* s);
/* With a skin: blocks of steps that ran in the exact mode (a list check
 * before every step, chosen on the device when particles are fast for the
 * skin) since the simulation was created. */
int blaze_num_exact_blocks(blaze_sim* s);
/* Wait for the stream; returns the accumulated status (see Part 1). */
int blaze_sync(blaze_sim* s);
int blaze_num_current(blaze_sim* s);
int blaze_num_rebuilds(blaze_sim* s);
int blaze_update_wobj(blaze_sim* s, const WOBJ* w, int n_w);
int blaze_update_dobj(blaze_sim* s, const DOBJ* d, int n_d);
/* Turn the volume objects attached to the drum (is_attached_DWorld) by
 * rad_per_step about the axis through (about_x, about_y) parallel to z
 * before every step, on the device, as the mill driver's
 * Rotate_VolObject_Inc does on the host before each Device_DEM_UpdateSim
 * (Processing_Mills.h:4-75, main.cpp:113-124): vertices and centre of mass
 * turned, face centroids, normals and areas recomputed, in its FP32
 * operation order with the host's cosf / sinf of the angle.  on = 0 stops. */
int blaze_set_dobj_rotation(blaze_sim* s, float about_x, float about_y, float rad_per_step,
                            int on);
/* Move volume object `index` by its velocity times dt before every step,
 * after any turn, on the device, as Translate_VolObject does when the
 * reference's driver translates it (Processing_Mills.h:336-396,
 * main.cpp:176-180).  on = 0 stops. */
int blaze_set_dobj_translation(blaze_sim* s, int index, int on);
/* Turn the world objects marked is_rotating by rad_per_step about the axis
 * through (about_x, about_y) parallel to z before every step, on the
 * device, as Rotate_WObject_inc does (Processing_Mills.h:257-334,
 * main.cpp:151-164): face vertices turned, centroids, normals and areas
 * recomputed.  Moving walls switch off the per-cell wall lists. */
int blaze_set_wobj_rotation(blaze_sim* s, float about_x, float about_y, float rad_per_step,
                            int on);
/* The volume / world objects as they are now (moved ones included). */
int blaze_get_dobj(blaze_sim* s, DOBJ* d, int n_d);
int blaze_get_wobj(blaze_sim* s, WOBJ* w, int n_w);
/* Energy tallies (SimulationInfo::EnergyCalc): energy dissipated in
 * particle-particle, volume-object and world-object contacts since the
 * last reset, in Device_Get_Energy's units (tally x 1e-4), summed in FP64 in
 * a fixed order (the reference adds FP32 values with float atomics);
 * spheres and polyhedra. */
int blaze_get_energy(blaze_sim* s, double* e3);
/* Set the raw tallies (Device_Set_Tallys); NULL zeroes them. */
int blaze_set_energy(blaze_sim* s, const double* raw3);
/* Last step's forces (capture_forces=1), AoS float3 x6: particle-particle
 * (incl. gravity), wall, volume-object; translational then rotational. */
int blaze_get_forces(blaze_sim* s, float* f_pp, float* t_pp, float* f_w, float* t_w, float* f_l,
                     float* t_l);
/* Neighbour list of the last rebuild: nn[i], list[i*max_nbr + k]. */
int blaze_get_nlist(blaze_sim* s, uint* nn, uint* list);
/* Device pointers of the current state (SoA float4: pos+radius, vel+type,
 * angular velocity) and the CUDA stream the simulation runs on. */
int blaze_device_state(blaze_sim* s, void** pos4, void** vel4, void** angv4, void** stream);
/* Headless replacement of the reference's OpenGL view (Graphics.h draws
 * positions and, for polyhedra, orientations every frame): waits for the
 * stream, then returns device pointers to the current step's positions as
 * float4 (x, y, z, radius; polyhedra: centre of mass) and orientations as
 * float4 (w, x, y, z; NULL for spheres), in memory order, and the number of
 * entries n (particles removed since the last re-sort are parked far
 * outside the world).  The pointers stay valid until the next step or
 * state change; read them on `stream` or after this call.  Returns the
 * status like blaze_sync. */
int blaze_device_view(blaze_sim* s, const void** pos4, const void** ornt4, int* n, void** stream);
/* Kernel launches the last blaze_step enqueued unconditionally (gate and
 * step kernels; graph re-sort bodies are counted by blaze_rebuild_kernels
 * per re-sort). */
int blaze_last_launches(blaze_sim* s);
/* Kernels one re-sort + neighbour-list rebuild launches. */
int blaze_rebuild_kernels(blaze_sim* s);
/* Per-phase CUDA-event timing of subsequent steps (on/off), and the totals
 * since it was switched on: re-sort + neighbour-list phase and the fused
 * step kernel, in ms, with the number of steps timed. */
int blaze_set_profile(blaze_sim* s, int on);
int blaze_profile(blaze_sim* s, float* ms_rebuild, float* ms_step, int* n_steps);
/* Drop the last world object (the silo hatch), as Device_OpenHatch does
 * without re-uploading the objects. */
int blaze_open_hatch(blaze_sim* s);
/* State files in the reference's format (Output_SystemState,
 * FileIO.h:12-315): what the writer takes from the driver's globals. */
typedef struct blaze_state_header {
  int detail;          /* Specfication_Detail 1..5 */
  int sim_type;        /* 0 general, 1 ball mill, 2 silo */
  int rotating_wobj;   /* general run with a rotating world object */
  int particle_type;   /* 0 spheres, 1 polyhedra */
  int fill_start;      /* the start file a mill fill writes (zeroed mill line) */
  int revflag;         /* mill: 1 at the end of a revolution */
  int rev_number;      /* mill: the revolution counter */
  int num_rem;         /* silo: particles left */
  int rot_steps;       /* rotating world object: steps turned */
  int steps_per_rev;   /* mill: steps per revolution (power line) */
  double time;         /* simulated time, s */
  double rot_angle;    /* mill / rotating world object: angle turned */
  float energy[5];     /* mill: particle, lifter, drum, normal, shear */
  float hatch_height;  /* silo: the speed statistics count particles above it */
  float dt;            /* time step (power line) */
} blaze_state_header;
/* Write host arrays (memory order, n = particles in the run; quat4 w first;
 * pobj for detail 5) as the reference's writer does.  No GPU needed. */
int blaze_write_state_arrays(const char* path, const blaze_state_header* h, int n,
                             const float* pos3, const float* quat4, const float* vel3,
                             const float* avel3, const float* acc3, const uint* type,
                             const int* pid, const POBJ* pobj, int n_p);
/* The simulation's current state to `path` (accelerations are not kept:
 * detail 4's acceleration column is 0). */
int blaze_write_state(blaze_sim* s, const char* path, const blaze_state_header* h);
/* Silo_Stats (main.cpp:253-280), on the device: *count = the particles of
 * the current run (memory positions [0, n_cur)) above `height`, the hatch
 * height; particles removed since the last re-sort still sit in that range
 * at the parking position and count, as in the reference.  Waits for the
 * stream; returns the status like blaze_sync. */
int blaze_count_above(blaze_sim* s, float height, int* count);
/* The driver's result files, one line appended per call, as main.cpp
 * writes them (ostream defaults).  FlowRate.dat (main.cpp:142): time and
 * the percentage discharged, (n0 - remaining) / (float) n0 * 100.
 * Results.dat (main.cpp:74-82): per revolution the total, particle, lifter
 * and drum power from Device_Get_Energy's three values over
 * steps_per_rev * dt.  No GPU needed.  0 ok, -1 bad argument, -3 I/O. */
int blaze_write_flow_line(const char* path, double time, int n0, int remaining);
int blaze_write_power_line(const char* path, double time, const float* energy3, int steps_per_rev,
                           float dt);
/* Self-check of the step's shared-reciprocal division against IEEE
 * division on the GPU: components that differ over n random triples
 * (0 expected), -1 on error. */
long long blaze_check_division(long long n, unsigned long long seed);
/* The simulation behind Part 1 (NULL before Device_Set_SimulationData). */
blaze_sim* blaze_default_sim(void);

/* Contact list of one set of spheres, computed without allocating any
 * device memory.  No counterpart in the reference.
 *
 * For callers that may not allocate: a solver that calls the broad phase
 * between its own kernels (coupled CFD-DEM, FEM) cannot afford cudaMalloc /
 * cudaFree, which synchronise the whole device, and many such hosts own all
 * device memory through their own pool.  The working memory is a fixed
 * array inside the library (about 5.8 MB, held on every GPU that loads the
 * library until the process exits), which limits a call to 65,536 spheres
 * and 262,144 hash-table entries; larger calls return -3 with a message.
 *
 * Same broad phase as the step: cell keys from si->worldOrigin, cellSize and
 * num_NNCells, stable sort by cell, and every pair with
 * |xi - xj| - (ri + rj) < skin from the 27 surrounding cells.  The list
 * holds every such pair only when each cell edge is at least 2 r_max + skin
 * (a pair further apart than one cell edge is not searched); a sphere with
 * 2 r + skin above the smallest edge raises status 128.
 *   pos4    device, n x (x, y, z, radius) floats, every particle live
 *   perm    device, n: sorted slot k holds input particle perm[k]
 *   nn      device, n: neighbour count of sorted particle i (<= max_nbr)
 *   list    device, max_nbr * n, slot-major: list[k * n + i] is the k-th
 *           neighbour of sorted particle i, as a sorted slot
 *   status  device, 1 word (may be NULL): status bits (1 overflow, 2 outside
 *           the grid, 128 cells too small for the skin)
 *   stream  cudaStream_t the work is enqueued on (NULL: default stream)
 * Returns 0 once the work is enqueued, -1 for a bad argument, -3 beyond the
 * size limit, -(1000 + cudaError_t) for a CUDA error.  The first call on
 * each device looks up the array's device address; make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int blaze_contact_list_static(const float* pos4, int n, const SimulationInfo* si, float skin,
                              int max_nbr, int* perm, uint* nn, uint* list, uint* status,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif
