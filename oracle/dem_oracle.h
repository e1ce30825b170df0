/*
 * dem_oracle.h -- CPU restatement of the per-step sphere DEM path, compiled
 * twice from dem_oracle.c: with DEM_REAL=float it follows the reference's
 * FP32 operation order exactly and is pinned bit-for-bit against the
 * reference's own kernels compiled on the host; with DEM_REAL=double it is
 * the FP64 oracle the GPU's FP32 error is stated against.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it as the checker; the product never does.
 *
 * All state crosses this interface as double arrays (the float build
 * converts exactly).  Particle order is the current memory order, i.e. the
 * cell-sorted order of the last step, as in the reference.
 */
#ifndef DEM_ORACLE_H_
#define DEM_ORACLE_H_

#include "../include/blaze_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dem_oracle dem_oracle;

/* Contact laws beyond the reference's (the reference law is law 0). */
typedef struct dem_law {
  int model;        /* 0 reference linear + velocity friction (Collision_Response.cuh)
                       1 linear spring-dashpot + tangential history spring + Coulomb cap
                       2 Hertz-Mindlin (no-slip) + history + Coulomb cap                  */
  double kt_ratio;  /* model 1: tangential stiffness / normal stiffness (2/7)               */
  double youngs;    /* model 2: Young's modulus, kg/(cm s^2)                                */
  double poisson;   /* model 2: Poisson ratio                                               */
  double restitution; /* models 1/2: coefficient of restitution used for the damping      */
  double mu;        /* models 1/2: Coulomb friction coefficient                             */
  double mu_roll;   /* models 1/2: rolling friction coefficient (constant-torque model)    */
  double skin;      /* neighbour list skin, cm (0 = contacts only, rebuilt every step)     */
  int max_nbr;      /* neighbour slots per particle (reference: 32)                        */
} dem_law;

dem_oracle* dem_create(const SimulationInfo* si, const WOBJ* w, int n_w, const POBJ* p, int n_p,
                       const DOBJ* d, int n_d);
void dem_destroy(dem_oracle* o);
void dem_set_law(dem_oracle* o, const dem_law* law);
void dem_set_cylinder_rotation(dem_oracle* o, int on);
void dem_set_state(dem_oracle* o, const double* pos3, const double* vel3, const double* avel3,
                   const unsigned* type, const int* pid);
/* Per-particle radius/mass/inverse-inertia overrides (polydisperse runs);
 * NULL restores the per-type values of the particle objects. */
void dem_set_particle_props(dem_oracle* o, const double* radius, const double* mass);
int dem_step(dem_oracle* o, int nsteps);
int dem_num_current(const dem_oracle* o);
void dem_get_state(const dem_oracle* o, double* pos3, double* vel3, double* avel3, unsigned* type,
                   int* pid);
/* Forces of the last step before integration: particle-particle (incl.
 * gravity), wall and volume-object parts, translational and rotational. */
void dem_get_forces(const dem_oracle* o, double* f_pp, double* t_pp, double* f_w, double* t_w,
                    double* f_l, double* t_l);
/* Contact list of the last rebuild (slot-major view: list[i*max_nbr+k]). */
void dem_get_nlist(const dem_oracle* o, unsigned* nn, unsigned* list);
/* Status bits of the last step (same bit meanings as the product's). */
int dem_status(const dem_oracle* o);
/* Energy dissipation tallies (particle, volume object, surface), J. */
void dem_get_energy(const dem_oracle* o, double* e3);
void dem_update_wobj(dem_oracle* o, const WOBJ* w, int n_w);
void dem_update_dobj(dem_oracle* o, const DOBJ* d, int n_d);
/* Triangle-mesh walls (law/geometry extension): n triangles, 9 values each. */
void dem_set_mesh(dem_oracle* o, const double* tri9, int n_tri, double kn, double cn, double mu);

#ifdef __cplusplus
}
#endif
#endif
