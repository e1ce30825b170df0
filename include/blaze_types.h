/*
 * blaze_types.h -- plain-old-data types that cross the simulation-step
 * boundary, byte-identical to the reference's own definitions so that a
 * caller's existing project-input code (KSimulationData) can hand its objects
 * to this library unchanged.
 *
 * Layouts follow, field for field:
 *   SimulationInfo  V_02_2015/src/DataStructures/KSimulationObjects.h:104-152
 *   InitConfig      KSimulationObjects.h:158-182
 *   Surface         KSimulationObjects.h:241-251
 *   PP_Parms        KSimulationObjects.h:261-267
 *   POBJ            KSimulationObjects.h:272-304
 *   DOBJ            KSimulationObjects.h:318-342
 *   Macro_Cylinder  KSimulationObjects.h:350-363
 *   WOBJ            KSimulationObjects.h:370-381
 *   Quaterion       V_02_2015/src/Utilities/Common/Types.h:15-21
 * Capacities (8 world objects x 16 faces, 8 particle types with a 6-entry
 * pair table, 32 volume objects) are the reference's; the tests check
 * sizeof/offsetof against the reference's headers compiled on the host.
 *
 * If the reference's KSimulationObjects.h / Types.h were included first
 * (as KDevice.h does), their definitions are used and this file adds
 * nothing.
 */
#ifndef BLAZE_TYPES_H_
#define BLAZE_TYPES_H_

#include <vector_types.h>

#ifdef __cplusplus
#include <cstdbool>
#else
#include <stdbool.h>
#endif

#ifndef TYPES_H_
#define TYPES_H_
typedef unsigned int uint;
typedef unsigned short ushort;
typedef struct Quaterion {
  float w; /* scalar part */
  float x;
  float y;
  float z;
} Quaterion;
#endif

#ifndef KSIMULATIONOBJECTS_H_
#define KSIMULATIONOBJECTS_H_

typedef enum Sim_Type { general = 0, ballmill = 1, silo = 2 } Sim_Type;
typedef enum SurfaceType { plane = 0, cylinder = 1 } SurfaceType;

typedef struct SimulationInfo {
  int particle_type; /* 0 spheres, 1 polyhedra */
  int Num_Particles;
  int Num_ParticleObjects;
  int* Num_ParticlesPerObject;
  int Num_WorldObjects;
  int TotnumCells;
  bool Rotation;
  bool Mode2D;
  bool EnergyCalc;
  bool isMillSim;
  bool Kill_Particles;
  float InitalDelta_t;
  float MillRotVel;
  float Global_VisDamp;
  float Roll_Res;
  float Silo_Kill_Height;
  float Vel_Limit;
  float DObject_CylinderBoundR;
  int3 num_NNCells;
  float3 Force_Field;
  float3 worldOrigin;
  float3 cellSize;
  float3 cent;
  float3 Vel_Limit_Bounds;
  float3 max_size;
  Sim_Type Simulation_Type;
  int Integration_Type;
  bool use_symmetry;
  bool sphere_orient;
  bool dobject_hasVertex;
  bool Rotating_WObject;
  bool use_hist;
  int unit_test;
} SimulationInfo;

typedef struct InitConfig {
  int3 num;
  float3 space;
  float3 start;
  float3 p_size[16];
  bool is_spheres;
  bool use_file;
  int grid_type;
  float3 launch_Vel;
  float3 fill_plane_start;
  float3 fill_plane_end;
  float3 velocity[12];
  float3 position[12];
  float3 ang_vel[12];
  bool DebugFlag;
  int use_device;
  bool multi_gpu;
  int threads_perBlock;
} InitConfig;

typedef struct Edge_Def {
  uint point_vindex[2];
} Edge_Def;

typedef struct Surface {
  int num_vertex;
  int vertex_Order[8];
  float area;
  float3 normal;
  float3 centroid;
  float Tol; /* point-in-polygon area tolerance, percent */
} Surface;

typedef struct PP_Parms {
  float Kn;
  float Cn;
  float Fric_static;
  float Fric_kinetic;
} PP_Parms;

typedef struct POBJ {
  float radius; /* cm */
  float mass;   /* kg */
  float3 COM;
  int num_vertex;
  float3 Local_Vertex[32];
  int num_edges;
  Edge_Def edge[32];
  int num_faces;
  Surface face[32];
  float InertiaT[9];
  float3 vertex[32];
  PP_Parms PP[6];
  float surface_Kn;
  float surface_Cn;
  float surface_Fric_static;
  float surface_Fric_kinetic;
  float Dsurface_Kn;
  float Dsurface_Cn;
  float Dsurface_Fric_static;
  float Dsurface_Fric_kinetic;
} POBJ;

typedef struct DOBJ {
  uint btype;
  float3 Axis;
  float boundR;
  float3 COM;
  int num_vertex;
  float3 vertex[8];
  int num_faces;
  Surface faces[3];
  int num_edges;
  Edge_Def edge[4];
  float3 velocity;
  bool is_attached_DWorld;
  bool is_translating;
} DOBJ;

typedef struct Macro_Cylinder {
  float height;
  float radius;
  bool has_top_cap;
  bool has_bot_cap;
  float3 normal_cyl;
  float3 normal_top_cap;
  float3 normal_bot_cap;
  float3 center_top_cap;
  float3 center_bot_cap;
  float3 AXIS;
} Macro_Cylinder;

typedef struct WOBJ {
  SurfaceType surface_type;
  int num_surfaces;
  Surface surfaces[16];
  int num_vertex;
  float3 vertex[16];
  bool is_rotating;
  Macro_Cylinder cyl_geo;
} WOBJ;

#endif /* KSIMULATIONOBJECTS_H_ */

#endif /* BLAZE_TYPES_H_ */
