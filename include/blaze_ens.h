/*
 * blaze_ens.h -- C ABI of DEM ensembles in libblaze_b200.so: many independent
 * sphere systems of uneven size stepped together on one GPU, with contact
 * laws the reference does not have.
 *
 * The reference runs one system per process (DeviceInterface.cu:1499-1816)
 * with a linear spring-dashpot and a velocity-proportional tangential force
 * (Collision_Response.cuh:374-494).  An ensemble keeps the reference's step
 * structure -- hash, stable sort by cell (BroadPhase.cuh:75-117), reorder and
 * cell table (BroadPhase.cuh:126-325), 27-cell neighbour search
 * (BroadPhase.cuh:402-513), per-particle force gather and symplectic Euler
 * (DEM_Kernels_Compute.cuh:620-729, Integration.cuh:6-184) -- over all
 * systems at once, with
 *   - keys prefixed by the system (a particle only meets its own system),
 *   - a Verlet list with skin, rebuilt when any particle has moved half of it,
 *   - the linear (kn, kt) or Hertz-Mindlin (E, nu) normal/tangential spring
 *     with restitution damping, a tangential history spring capped by
 *     Coulomb friction, and rolling friction,
 *   - walls: planes, cylinders (particles inside) and triangle meshes.
 * Status codes as in blaze_dem.h (0 ok, >0 status bits, <0 errors).
 * Units are the reference's: cm, kg, s.
 */
#ifndef BLAZE_ENS_H_
#define BLAZE_ENS_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct blaze_ens blaze_ens;

/* BLAZE_LAW_REFERENCE: the reference's own sphere law and step
 * (Collision_Response.cuh:374-494 and 4-109, Integration.cuh:6-184): linear
 * spring-dashpot without history, the tangential force
 * mu_k (m_a + m_b) / (40 dt) |v_t| / |v_rel| against v_t, plane walls as the
 * reference's faces, its contact test and penetration (+1e-5 cm), with the
 * parameters its parser derives for a particle object (KSimulationData.cpp:
 * 955-1047, 1096) formed per particle from the radius: kn, the damping from
 * the restitution and the (reduced) mass, mu (pairs, kinetic), mu_wall
 * (walls, static), mu_roll as the reference's rolling resistance (RollRes).
 * Plane walls only; kt_ratio, youngs and poisson are not read. */
enum { BLAZE_LAW_LINEAR = 1, BLAZE_LAW_HERTZ_MINDLIN = 2, BLAZE_LAW_REFERENCE = 3 };
enum { BLAZE_WALL_PLANE = 0, BLAZE_WALL_TRIANGLE = 1, BLAZE_WALL_CYLINDER = 2 };

typedef struct blaze_wall {
  int kind;     /* BLAZE_WALL_* */
  float p[10];  /* plane:    p[0..2] unit normal pointing into the domain, p[3] = d
                 *           (points x of the plane have n . x = d)
                 * triangle: p[0..8] the three vertices
                 * cylinder: p[0..2] a point on the axis, p[3..5] unit axis,
                 *           p[6] radius (particles move inside)            */
} blaze_wall;

typedef struct blaze_system {
  int n;              /* particles; systems are consecutive in the state arrays */
  float origin[3];    /* hash grid origin, cm */
  float cell;         /* cubic cell edge, cm; must be >= 2 r_max + skin */
  int ncells[3];
  float gravity[3];   /* cm/s^2 */
  float density;      /* kg/cm^3: m = density 4/3 pi r^3, I = 0.4 m r^2 */
  float kn;           /* linear law: normal stiffness, kg/s^2 */
  float kt_ratio;     /* linear law: tangential / normal stiffness (e.g. 2/7) */
  float youngs;       /* Hertz-Mindlin: Young's modulus, kg/(cm s^2) (1 Pa = 0.01) */
  float poisson;      /* Hertz-Mindlin: Poisson ratio */
  float restitution;  /* normal coefficient of restitution, (0, 1] */
  float mu;           /* Coulomb friction, particle-particle */
  float mu_wall;      /* Coulomb friction, particle-wall */
  float mu_roll;      /* rolling friction coefficient (0: none) */
  int wall0, nwalls;  /* planes and cylinders of this system: walls[wall0 .. +nwalls) */
  int tri0, ntris;    /* triangles of this system: walls[tri0 .. +ntris) */
  /* A turning drum: the system's triangles and cylinders turn at rot_omega
   * (rad/s, right-handed about rot_axis, a unit vector, through rot_point),
   * from their given positions at the last blaze_ens_set_state.  Their
   * surfaces move with the turn (the contact laws see the relative
   * velocity, and the drum's spin in the rolling friction).  Cylinders must
   * be coaxial with the turn (they stay in place); planes normal to the
   * axis (end plates) stay in place and their surfaces move; other planes
   * stand still.
   * The turn is advanced on the device after every step by the constant
   * increment (cos, sin of rot_omega dt in float) and renormalised.
   * rot_omega 0: nothing turns. */
  float rot_point[3];
  float rot_axis[3];
  float rot_omega;
} blaze_system;

typedef struct blaze_ens_options {
  int law;             /* BLAZE_LAW_LINEAR, BLAZE_LAW_HERTZ_MINDLIN or BLAZE_LAW_REFERENCE */
  float dt;            /* s */
  float skin;          /* Verlet skin, cm, > 0 */
  int max_nbr;         /* neighbour / history slots per particle, 1..32 */
  int use_graph;       /* 1: steps run as CUDA graphs (re-sort in a conditional node);
                        * 2: persistent stepping: one graph per call whose WHILE
                        *    node runs rounds of (re-sort if asked, then one
                        *    cooperative kernel that runs the steps up to the
                        *    next re-sort with a grid barrier between steps;
                        *    a barrier wait that gives up after 2 s raises
                        *    status 16); not with capture_forces */
  int capture_forces;  /* 1: keep each step's contact force and torque per particle */
  int block;           /* threads per block of the step kernel: 64, 128, 256 or 512 */
} blaze_ens_options;

/* law 1, dt 1e-5, skin 0.02, max_nbr 32, use_graph 1, capture_forces 0, block 256 */
void blaze_ens_default_options(blaze_ens_options* o);

int blaze_ens_create(blaze_ens** out, const blaze_system* systems, int nsys,
                     const blaze_wall* walls, int nwalls, const blaze_ens_options* opt);
int blaze_ens_destroy(blaze_ens* e);
/* Host arrays of all systems concatenated in system order: positions (3 per
 * particle), radii, velocities and angular velocities (may be NULL: zero).
 * Clears every contact history.  Radii must satisfy 2 r + skin <= cell. */
int blaze_ens_set_state(blaze_ens* e, const float* pos3, const float* radius, const float* vel3,
                        const float* avel3);
/* Current memory order (sorted by system and cell); sys[i] is the system of
 * entry i and pid[i] its index in the set_state arrays.  NULL skips an array. */
int blaze_ens_get_state(blaze_ens* e, float* pos3, float* radius, float* vel3, float* avel3,
                        int* sys, int* pid);
/* Self-check of persistent stepping's bounded barrier wait: two blocks wait
 * at a barrier counted for three, which nothing completes; after the 2 s
 * limit every block gives up and returns.  Returns the status words raised
 * (16 expected: a bounded device wait gave up), <0 on a CUDA error; the
 * context stays usable. */
int blaze_ens_check_barrier_timeout(void);
/* Enqueue nsteps steps on the ensemble's stream. */
int blaze_ens_step(blaze_ens* e, int nsteps);
/* Wait for the stream; the status bits raised since the state was set. */
int blaze_ens_sync(blaze_ens* e);
/* New law parameters (same sizes, grids and walls as at creation). */
int blaze_ens_set_params(blaze_ens* e, const blaze_system* systems);
/* capture_forces: contact force and torque of the last step (gravity not
 * included), 3 floats per particle, current memory order. */
int blaze_ens_get_forces(blaze_ens* e, float* force3, float* torque3);
int blaze_ens_num_rebuilds(blaze_ens* e);
/* Device pointers of the current state (float4 pos+radius, vel+bits,
 * angular velocity+path) and the ensemble's CUDA stream. */
int blaze_ens_device_state(blaze_ens* e, void** pos4, void** vel4, void** angv4, void** stream);
/* Kernels launched by the last blaze_ens_step that always run (re-sorts are
 * counted by blaze_ens_rebuild_kernels each). */
int blaze_ens_last_launches(blaze_ens* e);
int blaze_ens_rebuild_kernels(blaze_ens* e);
/* Profiling: while on, blaze_ens_step runs plain steps, each waiting for the
 * device, and adds their device time by phase: the re-sort (with the gate;
 * zero-work launches when no re-sort is due), the polyhedron geometry, the
 * polyhedron step, the sphere step.  Turning it on clears the sums. */
int blaze_ens_set_profile(blaze_ens* e, int on);
/* ms4: the four sums in ms; steps: the plain steps they cover. */
int blaze_ens_profile(blaze_ens* e, float* ms4, int* steps);

/* ------------------------------------------------------------- polyhedra
 * Convex polyhedra among the spheres of a system (the mixed charge of the
 * ball mill: steel balls and rocks).  The reference runs either spheres or
 * polyhedra, never both (KSimulationData.cpp:129-141).
 *
 * A shape is a closed convex hull of 4..16 vertices and 2 V - 4 triangular
 * faces in its body frame, centre of mass at the origin, faces
 * counter-clockwise seen from outside, with its density.  A polyhedron
 * meets
 *   spheres     at the closest point of its hull to the sphere's centre,
 *   polyhedra   along the axis of least penetration of the separating-axis
 *               test (face normals of both hulls, cross products of the edge
 *               pairs that form a face of the Minkowski difference), a face
 *               preferred unless an edge pair is clearly shallower,
 *   triangles   the same test with the triangle as a flat hull; contacts
 *               along a triangle's face normal all count, coplanar ones
 *               once (the deepest), and without one only the deepest
 *               other contact counts,
 *   planes      at its deepest vertex,
 * all formed in FP64 from the FP32 state; the contact point is the mean of
 * the penetrating vertices weighted by their depths, or the midpoint of two
 * crossing edges.  The law
 * is the linear law with tangential history and Coulomb cap on the contact
 * point's relative velocity, without rolling friction; a polyhedron
 * integrates Euler's equations in its body frame and its orientation as a
 * unit quaternion.  Systems holding polyhedra: linear law, plane and
 * triangle walls (no cylinders), 2 r_bound + skin <= cell; per
 * polyhedron at most 64 neighbours, 16 wall contacts and 32 touching
 * triangles a step (beyond them status 1); not with persistent stepping
 * (use_graph 2 steps as 1) nor reverse mode. */
typedef struct blaze_shape {
  int nverts;            /* 4 .. 16 */
  int nfaces;            /* 2 nverts - 4 */
  float density;         /* kg/cm^3 */
  float verts[16 * 3];   /* body frame, cm, centre of mass at the origin */
  int faces[28 * 3];     /* vertex indices per face, counter-clockwise seen from outside */
} blaze_shape;

/* Mass (kg), centre of mass (cm), inertia tensor about the centre of mass
 * (kg cm^2, row-major) and bounding radius about the origin (cm, rounded
 * up) of a shape, in FP64 from its faces; no device needed.  Returns -1 for
 * a shape that is not a closed, outward-oriented convex hull of the sizes
 * above. */
int blaze_shape_mass_properties(const blaze_shape* s, double* mass, double* com3,
                                double* inertia9, float* rbound);

/* Right after blaze_ens_set_state (before any step): the particles with
 * shape_of[i] >= 0 (caller order) are polyhedra of shapes[shape_of[i]] with
 * orientation quat4[4 i ..] = (w, x, y, z) (normalised here); their radius
 * in the state becomes the shape's bounding radius.  A later set_state
 * leaves only spheres.  Returns -1 on a shape or system the rules above
 * exclude. */
int blaze_ens_set_polyhedra(blaze_ens* e, const blaze_shape* shapes, int nshapes,
                            const int* shape_of, const float* quat4);
/* Orientations in the current memory order (4 floats per particle, w x y z;
 * spheres 1 0 0 0). */
int blaze_ens_get_orientations(blaze_ens* e, float* quat4);

/* ------------------------------------------------------------ reverse mode
 * Gradients of a loss of the final state with respect to the initial state
 * and the law constants, by the discrete adjoint of the step (linear law
 * with tangential history and Coulomb cap, plane walls, no rolling
 * friction).  The forward keeps a checkpoint of the full state every
 * `segment` steps and records the trailing segments into a tape; the
 * backward walks the tape back segment by segment, recomputing from its
 * checkpoint each segment the tape no longer holds.  Derivatives are those of the branch
 * each contact took (contact or not, stick or slip). */
typedef struct blaze_ens_adj blaze_ens_adj;

int blaze_ens_adj_create(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment);
/* The same with a tape budget.  The tape is one arena holding, per recorded
 * step, the input state and history mask (68 B per particle) and the step's
 * active histories, and per re-sort the new list.  The forward records the
 * trailing segments that fit as it runs (a ring of segments), and the
 * backward recomputes only the others.
 *   tape_bytes == 0: one segment, with room for the most it can take (every
 *                    list slot an active history, a re-sort every step);
 *   tape_bytes  > 0: an arena of that many bytes;
 *   tape_bytes  < 0: 96 % of the device memory the reverse mode's other
 *                    buffers leave free, less 4 GiB.
 * Returns -2 when the arena cannot hold one segment's states; a backward
 * whose recomputed segment does not fit the arena also returns -2. */
int blaze_ens_adj_create_ex(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment,
                            long long tape_bytes);
/* The same with the arena size given in bytes. */
int blaze_ens_adj_create_tape(blaze_ens_adj** out, blaze_ens* e, int nsteps, int segment,
                              unsigned long long arena_bytes);
/* nsteps steps from the ensemble's current state, with checkpoints; the
 * ensemble then holds the final state (read it with blaze_ens_get_state). */
int blaze_ens_adj_forward(blaze_ens_adj* a);
/* Cotangents of the final state (3 floats per particle, final memory order;
 * NULL for zero) -> cotangents of the initial state (its memory order; NULL
 * skips) and of the law constants of every system (nsys x 5 doubles: kn,
 * kt, 2 beta, mu, mu_wall; beta = -ln e / sqrt(ln^2 e + pi^2)).  Leaves the
 * ensemble at an intermediate state: set the state again before stepping. */
int blaze_ens_adj_backward(blaze_ens_adj* a, const float* gpos, const float* gvel,
                           const float* gavel, float* gpos0, float* gvel0, float* gavel0,
                           double* gconst);
/* The reverse sweep over the last `window` steps only (truncated
 * backpropagation): the law-constant cotangents of those steps, and the
 * cotangents of the state at step nsteps - window (that step's memory
 * order; NULL skips), the earlier state held fixed.  Over long horizons
 * the full discrete adjoint of dense granular flow grows exponentially
 * with the horizon (the dynamics is chaotic: the derivative along the
 * contact onsets and stick/slip states taken, measured about 5 % per step
 * at dt = 1e-5 s), so the full backward of a 3,000-step run overflows FP32;
 * a window keeps the gradient bounded and local.  window = nsteps is
 * blaze_ens_adj_backward. */
int blaze_ens_adj_backward_window(blaze_ens_adj* a, int window, const float* gpos,
                                  const float* gvel, const float* gavel, float* gpos_w,
                                  float* gvel_w, float* gavel_w, double* gconst);
/* Device time of the last backward call by phase, ms: restoring the
 * checkpoints, recomputing the segments into the tape, the reverse sweep. */
int blaze_ens_adj_profile(blaze_ens_adj* a, float* ms_restore, float* ms_record,
                          float* ms_reverse);
/* Arena size, how many segments the last forward left on the tape (the
 * backward recomputes the others from their checkpoints), and the most pool
 * bytes (histories and lists) one recorded segment has taken so far. */
int blaze_ens_adj_tape_info(blaze_ens_adj* a, unsigned long long* arena_bytes, int* on_tape,
                            unsigned long long* pool_bytes_max);
int blaze_ens_adj_destroy(blaze_ens_adj* a);

#ifdef __cplusplus
}
#endif
#endif
