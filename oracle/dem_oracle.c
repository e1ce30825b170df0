/*
 * dem_oracle.c -- CPU restatement of the reference's per-step sphere DEM path.
 * TEST INFRASTRUCTURE ONLY (see dem_oracle.h).
 *
 * Built twice: DEM_REAL=float reproduces the reference's FP32 arithmetic in
 * the reference's operation order (each function cites the lines it
 * follows; build flag -ffp-contract=off keeps a*b+c as two roundings, as the
 * reference's own expression order states it); DEM_REAL=double runs the same
 * algorithm in FP64.
 *
 * Step order: Device_DEM_UpdateSim, V_02_2015/src/Device/DeviceInterface.cu:1825-2513.
 */
#include "dem_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef DEM_REAL
#define DEM_REAL double
#endif
typedef DEM_REAL real;

#define IS_F32 (sizeof(real) == 4)
static inline real r_sqrt(real x) { return IS_F32 ? (real)sqrtf((float)x) : (real)sqrt((double)x); }
static inline real r_fabs(real x) { return IS_F32 ? (real)fabsf((float)x) : (real)fabs((double)x); }
static inline real r_floor(real x) { return IS_F32 ? (real)floorf((float)x) : (real)floor((double)x); }

typedef struct { real x, y, z; } v3;

static inline v3 mk(real x, real y, real z) { v3 r = {x, y, z}; return r; }
static inline v3 ff(float3 a) { return mk((real)a.x, (real)a.y, (real)a.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mulv(v3 a, real s) { return mk(a.x * s, a.y * s, a.z * s); }  /* float3*float */
static inline v3 smul(real s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }  /* float*float3 */
static inline v3 divs(v3 a, real s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 vmul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
/* Functions.cuh:198-372: dot is ((x*x + y*y) + z*z), length is sqrt(dot). */
static inline real dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline real len(v3 a) { return r_sqrt(dot(a, a)); }
static inline v3 cross(v3 a, v3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static const v3 Z3 = {0, 0, 0};

typedef struct { v3 trans, torque; } forces_t;
typedef struct {
  int is_collision;
  real dis;
  v3 contact_point, normal;
  int colltype;
} coll_t;

struct dem_oracle {
  SimulationInfo si;
  WOBJ w[8];
  POBJ p[8];
  DOBJ d[32];
  int n_w, n_p, n_d, num_wobj;
  int n_max, n_cur, num_dead, stepc, status;
  int cyl_rot;
  dem_law law;
  /* state (memory order) */
  v3 *pos, *vel, *avel;
  unsigned* type;
  int* pid;
  int* lift_type; /* Contact_Info.cont_type per particle */
  /* per-particle properties (radius/mass/inverse inertia by type unless overridden) */
  real *rad, *mass, *iinv;
  int props_override;
  /* scratch */
  uint32_t *key, *key2;
  int *idx, *idx2;
  uint32_t *cstart, *cend;
  size_t ncell;
  unsigned *nn, *nlist;
  v3 *f_pp, *t_pp, *f_w, *t_w, *f_l, *t_l;
  double e_pp, e_lift, e_surf;
  /* triangle mesh */
  double* tri;
  int n_tri;
  double mesh_kn, mesh_cn, mesh_mu;
};

enum { ST_LIST_OVERFLOW = 1, ST_OUT_OF_GRID = 2, ST_NONFINITE = 4 };

/* ------------------------------------------------------------------ grid */
/* SpatialDecomp_CalcGridPos / CalcGridHash, Collision_Detection_BroadPhase.cuh:20-50 */
static void grid_pos(const dem_oracle* o, v3 p, int g[3]) {
  g[0] = (int)r_floor((p.x - (real)o->si.worldOrigin.x) / (real)o->si.cellSize.x);
  g[1] = (int)r_floor((p.y - (real)o->si.worldOrigin.y) / (real)o->si.cellSize.y);
  g[2] = (int)r_floor((p.z - (real)o->si.worldOrigin.z) / (real)o->si.cellSize.z);
}
static uint32_t grid_hash(const dem_oracle* o, const int g[3]) {
  const int3 n = o->si.num_NNCells;
  return (uint32_t)((g[0] + g[2] * n.z) + (g[1] * n.x) * n.z);
}

/* ---------------------------------------------------------------- create */
dem_oracle* dem_create(const SimulationInfo* si, const WOBJ* w, int n_w, const POBJ* p, int n_p,
                       const DOBJ* d, int n_d) {
  if (!si || n_w < 0 || n_w > 8 || n_p < 1 || n_p > 8 || n_d < 0 || n_d > 32) return NULL;
  dem_oracle* o = (dem_oracle*)calloc(1, sizeof(dem_oracle));
  o->si = *si;
  if (n_w) memcpy(o->w, w, sizeof(WOBJ) * n_w);
  memcpy(o->p, p, sizeof(POBJ) * n_p);
  if (n_d) memcpy(o->d, d, sizeof(DOBJ) * n_d);
  o->n_w = n_w; o->n_p = n_p; o->n_d = n_d;
  o->num_wobj = si->Num_WorldObjects;
  const int n = si->Num_Particles;
  o->n_max = o->n_cur = n;
  o->law.model = 0;
  o->law.max_nbr = 32;
  o->pos = calloc(n, sizeof(v3)); o->vel = calloc(n, sizeof(v3)); o->avel = calloc(n, sizeof(v3));
  o->type = calloc(n, sizeof(unsigned)); o->pid = calloc(n, sizeof(int));
  o->lift_type = calloc(n, sizeof(int));
  for (int i = 0; i < n; ++i) o->lift_type[i] = -1;
  o->rad = calloc(n, sizeof(real)); o->mass = calloc(n, sizeof(real)); o->iinv = calloc(n, sizeof(real));
  o->key = calloc(n, 4); o->key2 = calloc(n, 4); o->idx = calloc(n, 4); o->idx2 = calloc(n, 4);
  const int3 nc = si->num_NNCells;
  /* Largest hash an in-grid cell can take, +1 (the reference sizes its
   * table ncx*ncy*ncz, which the hash formula exceeds when ncx < ncz). */
  long long hmax = (long long)(nc.x - 1) + (long long)(nc.z - 1) * nc.z +
                   (long long)(nc.y - 1) * nc.x * nc.z + 1;
  long long prod = (long long)nc.x * nc.y * nc.z;
  o->ncell = (size_t)(hmax > prod ? hmax : prod);
  o->cstart = malloc(o->ncell * 4); o->cend = malloc(o->ncell * 4);
  o->nn = calloc(n, 4);
  o->nlist = calloc((size_t)n * 32, 4);
  o->f_pp = calloc(n, sizeof(v3)); o->t_pp = calloc(n, sizeof(v3));
  o->f_w = calloc(n, sizeof(v3)); o->t_w = calloc(n, sizeof(v3));
  o->f_l = calloc(n, sizeof(v3)); o->t_l = calloc(n, sizeof(v3));
  return o;
}

void dem_destroy(dem_oracle* o) {
  if (!o) return;
  void* ps[] = {o->pos, o->vel, o->avel, o->type, o->pid, o->lift_type, o->rad, o->mass, o->iinv,
                o->key, o->key2, o->idx, o->idx2, o->cstart, o->cend, o->nn, o->nlist, o->f_pp,
                o->t_pp, o->f_w, o->t_w, o->f_l, o->t_l, o->tri};
  for (size_t k = 0; k < sizeof(ps) / sizeof(ps[0]); ++k) free(ps[k]);
  free(o);
}

void dem_set_law(dem_oracle* o, const dem_law* law) {
  o->law = *law;
  if (o->law.max_nbr < 1) o->law.max_nbr = 32;
  free(o->nlist);
  o->nlist = calloc((size_t)o->n_max * o->law.max_nbr, 4);
}

void dem_set_cylinder_rotation(dem_oracle* o, int on) { o->cyl_rot = on != 0; }

static void refresh_props(dem_oracle* o) {
  if (o->props_override) return;
  for (int i = 0; i < o->n_max; ++i) {
    const POBJ* P = &o->p[o->type[i] < 8 ? o->type[i] : 0];
    o->rad[i] = (real)P->radius;
    o->mass[i] = (real)P->mass;
    o->iinv[i] = (real)P->InertiaT[0];
  }
}

void dem_set_state(dem_oracle* o, const double* pos3, const double* vel3, const double* avel3,
                   const unsigned* type, const int* pid) {
  /* Set_PSystem_State, GPU_Memory_Transfer.cuh:377-418 */
  for (int i = 0; i < o->n_max; ++i) {
    o->pos[i] = mk((real)pos3[3 * i], (real)pos3[3 * i + 1], (real)pos3[3 * i + 2]);
    o->vel[i] = vel3 ? mk((real)vel3[3 * i], (real)vel3[3 * i + 1], (real)vel3[3 * i + 2]) : Z3;
    o->avel[i] = avel3 ? mk((real)avel3[3 * i], (real)avel3[3 * i + 1], (real)avel3[3 * i + 2]) : Z3;
    o->type[i] = type[i];
    o->pid[i] = pid[i];
  }
  refresh_props(o);
}

void dem_set_particle_props(dem_oracle* o, const double* radius, const double* mass) {
  if (!radius || !mass) {
    o->props_override = 0;
    refresh_props(o);
    return;
  }
  o->props_override = 1;
  for (int i = 0; i < o->n_max; ++i) {
    o->rad[i] = (real)radius[i];
    o->mass[i] = (real)mass[i];
    /* sphere inverse inertia 1/(0.4 m r^2), main.cpp:615-616 */
    o->iinv[i] = (real)1.0 / ((real)0.4 * o->rad[i] * o->rad[i] * o->mass[i]);
  }
}

void dem_update_wobj(dem_oracle* o, const WOBJ* w, int n_w) {
  if (n_w >= 0 && n_w <= 8) memcpy(o->w, w, sizeof(WOBJ) * n_w);
}
void dem_update_dobj(dem_oracle* o, const DOBJ* d, int n_d) {
  if (n_d >= 0 && n_d <= 32) memcpy(o->d, d, sizeof(DOBJ) * n_d);
}

void dem_set_mesh(dem_oracle* o, const double* tri9, int n_tri, double kn, double cn, double mu) {
  free(o->tri);
  o->tri = NULL;
  o->n_tri = 0;
  if (n_tri > 0) {
    o->tri = malloc(sizeof(double) * 9 * n_tri);
    memcpy(o->tri, tri9, sizeof(double) * 9 * n_tri);
    o->n_tri = n_tri;
  }
  o->mesh_kn = kn; o->mesh_cn = cn; o->mesh_mu = mu;
}

/* ------------------------------------------------------------- sort step */
/* Stable ascending sort of (key, index) by key -- the result
 * thrust::stable_sort_by_key gives (Collision_Detection_BroadPhase.cuh:110-117);
 * done here as an LSD counting sort, 8 bits per pass. */
static void stable_sort(dem_oracle* o, int n) {
  uint32_t kmax = 0;
  for (int i = 0; i < n; ++i) kmax = o->key[i] > kmax ? o->key[i] : kmax;
  static unsigned cnt[257];
  for (int shift = 0; shift < 32 && (kmax >> shift); shift += 8) {
    memset(cnt, 0, sizeof(cnt));
    for (int i = 0; i < n; ++i) cnt[((o->key[i] >> shift) & 255) + 1]++;
    for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
    for (int i = 0; i < n; ++i) {
      unsigned dst = cnt[(o->key[i] >> shift) & 255]++;
      o->key2[dst] = o->key[i];
      o->idx2[dst] = o->idx[i];
    }
    uint32_t* tk = o->key; o->key = o->key2; o->key2 = tk;
    int* ti = o->idx; o->idx = o->idx2; o->idx2 = ti;
  }
}

static void reorder(dem_oracle* o, int n) {
  /* Kernel_SortArrays + Kernel_SpatialDecomp_ReorderPDA (BroadPhase.cuh:126-268) */
  v3* tp = malloc(sizeof(v3) * n); v3* tv = malloc(sizeof(v3) * n); v3* tw = malloc(sizeof(v3) * n);
  unsigned* tt = malloc(4 * n); int* ti = malloc(4 * n); int* tl = malloc(4 * n);
  real *tr = malloc(sizeof(real) * n), *tm = malloc(sizeof(real) * n), *tI = malloc(sizeof(real) * n);
  for (int i = 0; i < n; ++i) {
    int s = o->idx[i];
    tp[i] = o->pos[s]; tv[i] = o->vel[s]; tw[i] = o->avel[s];
    tt[i] = o->type[s]; ti[i] = o->pid[s]; tl[i] = o->lift_type[s];
    tr[i] = o->rad[s]; tm[i] = o->mass[s]; tI[i] = o->iinv[s];
  }
  memcpy(o->pos, tp, sizeof(v3) * n); memcpy(o->vel, tv, sizeof(v3) * n);
  memcpy(o->avel, tw, sizeof(v3) * n); memcpy(o->type, tt, 4 * n); memcpy(o->pid, ti, 4 * n);
  memcpy(o->lift_type, tl, 4 * n);
  memcpy(o->rad, tr, sizeof(real) * n); memcpy(o->mass, tm, sizeof(real) * n);
  memcpy(o->iinv, tI, sizeof(real) * n);
  free(tp); free(tv); free(tw); free(tt); free(ti); free(tl); free(tr); free(tm); free(tI);
}

/* --------------------------------------------------------- contact list */
/* Kernel_BroadCollisionDetection_NonSymmetry + CollisionDetection_Filter_SphereNNCell
 * (Collision_Detection_BroadPhase.cuh:335-513): scan the clamped 3x3x3 block
 * in y, z, x order; keep j != i with |xi-xj| - (ri+rj) < skin. */
static void build_list(dem_oracle* o, int m) {
  const int cap = o->law.max_nbr;
  const real skin = (real)o->law.skin;
  const int3 nc = o->si.num_NNCells;
  for (int i = 0; i < m; ++i) {
    o->nn[i] = 0;
    if (o->pid[i] <= -1) continue;
    v3 pa = o->pos[i];
    int g[3];
    grid_pos(o, pa, g);
    int xs = -1, xe = 1, ys = -1, ye = 1, zs = -1, ze = 1;
    if (g[0] == 0) xs = 0;
    if (g[1] == 0) ys = 0;
    if (g[2] == 0) zs = 0;
    if (g[0] == nc.x - 1) xe = 0;
    if (g[1] == nc.y - 1) ye = 0;
    if (g[2] == nc.z - 1) ze = 0;
    unsigned cnt = 0;
    const real ra = o->rad[i];
    for (int y = ys; y <= ye; ++y)
      for (int z = zs; z <= ze; ++z)
        for (int x = xs; x <= xe; ++x) {
          int q[3] = {g[0] + x, g[1] + y, g[2] + z};
          uint32_t h = grid_hash(o, q);
          if (h >= o->ncell) continue;
          uint32_t s = o->cstart[h];
          if (s == 0xffffffffu) continue;
          uint32_t e = o->cend[h];
          for (uint32_t j = s; j < e; ++j) {
            if ((int)j == i) continue;
            real sep = len(sub(pa, o->pos[j])) - (ra + o->rad[j]);
            if (sep < skin) {
              if (cnt < (unsigned)cap) o->nlist[(size_t)i * cap + cnt] = j;
              else o->status |= ST_LIST_OVERFLOW;
              cnt++;
            }
          }
        }
    o->nn[i] = cnt < (unsigned)cap ? cnt : (unsigned)cap;
  }
}

/* ---------------------------------------------------- reference contact laws */
static real tally_gate(const dem_oracle* o) { return o->si.EnergyCalc ? 1 : 0; }

/* Collision_Response_Particle_Particle, Collision_Response.cuh:374-494 */
static forces_t law_pp_ref(dem_oracle* o, v3 rvel, v3 n, real pen, v3 ra, v3 rb, v3 wa, v3 wb,
                           const PP_Parms* pp, v3 va, v3 vb, real ma, real mb) {
  forces_t F;
  const real dt = (real)o->si.InitalDelta_t;
  v3 vn = smul(dot(rvel, n), n);
  real fn = (real)pp->Kn * pen;
  v3 fdiss = smul((real)pp->Cn, vn);
  F.trans = sub(smul(fn, n), fdiss);
  real etally = 0;
  if (o->si.EnergyCalc && dot(vn, vn) > 0) etally = (real)0.5 * len(fdiss) * len(vn) * dt;
  v3 vcpa = add(va, cross(wa, ra));
  v3 vcpb = add(vb, cross(wb, rb));
  v3 vcpna = smul(dot(vcpa, n), n);
  v3 vcpnb = smul(dot(vcpb, n), n);
  v3 vta = sub(vcpa, vcpna);
  v3 vtb = sub(vcpb, vcpnb);
  v3 vt = sub(vta, vtb);
  real mag = dot(vt, vt);
  v3 ft = Z3;
  if (mag > 0) {
    mag = r_sqrt(mag);
    real velf = dot(rvel, rvel);
    if (velf > 0) velf = r_sqrt(velf);
    else velf = 1;
    real tan_f = ((((real)0.5 * (ma + mb)) / dt) * (real)0.05) * (real)pp->Fric_kinetic * (mag / velf);
    ft = smul((real)-1.0 * tan_f, divs(vt, mag));
    if (o->si.EnergyCalc) o->e_pp += (double)(etally + len(ft) * mag * dt);
  } else if (o->si.EnergyCalc) {
    o->e_pp += (double)etally;
  }
  F.trans = add(F.trans, ft);
  F.torque = o->si.Rotation ? cross(ra, F.trans) : Z3;
  (void)tally_gate;
  return F;
}

/* Collision_Response_Particle_StaticSurface, Collision_Response.cuh:4-109 */
static forces_t law_static_surface(dem_oracle* o, v3 pvel, v3 n, real pen, v3 r, v3 w,
                                   const POBJ* P, real mass) {
  forces_t F;
  const real dt = (real)o->si.InitalDelta_t;
  v3 vn = smul(dot(pvel, n), n);
  real fn = (real)P->surface_Kn * pen;
  v3 fdiss = smul((real)P->surface_Cn, vn);
  F.trans = sub(smul(fn, n), fdiss);
  v3 fdir = divs(F.trans, len(F.trans));
  if (dot(fdir, n) < 0) {
    F.trans = smul(fn, n);
    fn = 0;
  } else {
    if (o->si.EnergyCalc && dot(vn, vn) > 0) fn = len(fdiss) * len(vn) * dt;
    else fn = 0;
  }
  v3 vt = sub(pvel, vn);
  v3 ft = Z3;
  if (o->si.Rotation) vt = add(vt, cross(w, r));
  real mag = dot(vt, vt);
  if (mag > 0) {
    mag = r_sqrt(mag);
    real velf = dot(pvel, pvel);
    if (velf > 0) velf = r_sqrt(velf);
    else velf = 1;
    real tan_f = ((real)0.05 * (mass / dt)) * ((real)P->surface_Fric_static * (mag / velf));
    ft = smul((real)-1.0 * tan_f, divs(vt, mag));
    if (o->si.EnergyCalc) o->e_surf += (double)(fn + len(ft) * mag * dt);
  } else if (o->si.EnergyCalc) {
    o->e_surf += (double)fn;
  }
  F.trans = add(F.trans, ft);
  F.torque = o->si.Rotation ? cross(r, F.trans) : Z3;
  return F;
}

/* Collision_Response_Particle_MovingSurface, Collision_Response.cuh:116-233 */
static forces_t law_moving_surface(dem_oracle* o, v3 n, real pen, v3 r, v3 w, const POBJ* P,
                                   v3 va, v3 vs, real mass) {
  forces_t F;
  const real dt = (real)o->si.InitalDelta_t;
  v3 rvel = sub(va, vs);
  v3 vn = smul(dot(rvel, n), n);
  real fn = (real)P->surface_Kn * pen;
  v3 fdiss = smul((real)P->surface_Cn, vn);
  F.trans = sub(smul(fn, n), fdiss);
  v3 fdir = divs(F.trans, len(F.trans));
  if (dot(fdir, n) < 0) {
    F.trans = smul(fn, n);
    fn = 0;
  } else {
    if (o->si.EnergyCalc && dot(vn, vn) > 0) fn = len(fdiss) * len(vn) * dt;
    else fn = 0;
  }
  v3 vcpa = add(va, cross(w, r));
  v3 vcpna = smul(dot(vcpa, n), n);
  v3 vta = sub(vcpa, vcpna);
  v3 vtb = sub(vs, smul(dot(vs, n), n));
  v3 vt = sub(vta, vtb);
  real mag = dot(vt, vt);
  v3 ft = Z3;
  if (mag > 0) {
    mag = r_sqrt(mag);
    real velf = dot(rvel, rvel);
    if (velf > 0) velf = r_sqrt(velf);
    else velf = 1;
    real tan_f = (real)P->surface_Fric_kinetic * (mag / velf);
    ft = smul((real)-1.0 * tan_f, divs(vt, mag));
    ft = mulv(ft, (mass / dt));
    ft = mulv(ft, (real)0.05);
    if (o->si.EnergyCalc) o->e_surf += (double)(fn + len(ft) * mag * dt);
  } else if (o->si.EnergyCalc) {
    o->e_surf += (double)fn;
  }
  F.trans = add(F.trans, ft);
  F.torque = o->si.Rotation ? cross(r, F.trans) : Z3;
  return F;
}

/* Collision_Response_Particle_VolumeObject, Collision_Response.cuh:241-363
 * (called with zero volume-object spin and lever, DEM_Kernels_Compute.cuh:206-216) */
static forces_t law_volume_object(dem_oracle* o, v3 n, real pen, v3 r, v3 w, const POBJ* P,
                                  v3 va, v3 vobj, real mass) {
  forces_t F;
  const real dt = (real)o->si.InitalDelta_t;
  v3 rvel = sub(va, vobj);
  v3 vn = smul(dot(rvel, n), n);
  real fn = (real)P->Dsurface_Kn * pen;
  v3 fdiss = smul((real)P->Dsurface_Cn, vn);
  F.trans = sub(smul(fn, n), fdiss);
  v3 fdir = divs(F.trans, len(F.trans));
  if (dot(fdir, n) < 0) {
    F.trans = smul(fn, n);
    fn = 0;
  } else {
    if (o->si.EnergyCalc && dot(vn, vn) > 0) fn = len(fdiss) * len(vn) * dt;
    else fn = 0;
  }
  v3 vcpa = add(va, cross(w, r));
  v3 vcpb = add(vobj, cross(Z3, Z3));
  v3 vcpna = smul(dot(vcpa, n), n);
  v3 vcpnb = smul(dot(vcpb, n), n);
  v3 vta = sub(vcpa, vcpna);
  v3 vtb = sub(vcpb, vcpnb);
  v3 vt = sub(vta, vtb);
  real mag = dot(vt, vt);
  v3 ft = Z3;
  if (mag > 0) {
    mag = r_sqrt(mag);
    real velf = dot(rvel, rvel);
    if (velf > 0) velf = r_sqrt(velf);
    else velf = 1;
    real tan_f = ((real)0.05 * (mass / dt)) * ((real)P->Dsurface_Fric_kinetic * (mag / velf));
    ft = smul((real)-1.0 * tan_f, divs(vt, mag));
    if (o->si.EnergyCalc) o->e_lift += (double)(fn + len(ft) * mag * dt);
  } else if (o->si.EnergyCalc) {
    o->e_lift += (double)fn;
  }
  F.trans = add(F.trans, ft);
  F.torque = o->si.Rotation ? cross(r, F.trans) : Z3;
  return F;
}

/* Collision_Response_EndPlate_Particle, Collision_Response.cuh:504-526 */
static forces_t law_end_plate(v3 rvel, v3 n, real pen, const POBJ* P) {
  forces_t F;
  v3 vn = smul(dot(rvel, n), n);
  v3 fdiss = smul((real)P->surface_Cn, vn);
  real fn = (real)P->surface_Kn * pen;
  F.trans = sub(smul(fn, n), fdiss);
  F.torque = Z3;
  return F;
}

/* ------------------------------------------------------- narrow phase: walls */
/* is_PointOnSurface, Utilities.cuh:20-53: polygon area by fan of triangles
 * about the point, compared with the face area within Tol percent. */
static int point_on_surface(int nv, const float3* vtx, const int* order, v3 pt, real sarea, real tol) {
  real area = 0;
  for (int i = 0; i < nv - 1; ++i) {
    v3 v1 = sub(pt, ff(vtx[order[i]]));
    v3 v2 = sub(pt, ff(vtx[order[i + 1]]));
    area = area + (real)0.5 * len(cross(v1, v2));
  }
  v3 v1 = sub(pt, ff(vtx[order[nv - 1]]));
  v3 v2 = sub(pt, ff(vtx[order[0]]));
  area = area + (real)0.5 * len(cross(v1, v2));
  return (r_fabs(area - sarea) / sarea) * (real)100.0 <= tol;
}

/* Collision_Detection_Sphere_Surface, Collision_Detection_Spheres.cuh:6-54 */
static coll_t sphere_surface(v3 p, real r, const Surface* s, const float3* vtx) {
  coll_t c;
  c.is_collision = 0;
  v3 n = ff(s->normal);
  v3 pt = sub(p, smul(r, n));
  c.dis = dot(n, sub(pt, ff(s->centroid)));
  if (c.dis < 0 && c.dis > -r) {
    c.dis = r_fabs(c.dis);
    v3 q = add(pt, mulv(n, c.dis));
    if (point_on_surface(s->num_vertex, vtx, s->vertex_Order, q, (real)s->area, (real)s->Tol)) {
      c.is_collision = 1;
      c.contact_point = pt;
      c.normal = n;
    }
  }
  return c;
}

/* Collision_Detection_Sphere_Plane, Collision_Detection_Spheres.cuh:63-100 */
static coll_t sphere_plane(v3 p, real r, v3 n, v3 cen) {
  coll_t c;
  c.is_collision = 0;
  v3 pt = sub(p, smul(r, n));
  c.dis = dot(n, sub(pt, cen));
  if (c.dis < 0 && c.dis > -r) {
    c.dis = r_fabs(c.dis);
    c.is_collision = 1;
    c.contact_point = pt;
    c.normal = n;
  }
  return c;
}

/* Collision_Detection_Sphere_Cylinder, Collision_Detection_Spheres.cuh:234-265 */
static coll_t sphere_cylinder(v3 p, real r, const Macro_Cylinder* cyl) {
  coll_t c;
  c.is_collision = 0;
  v3 pv = sub(vmul(p, ff(cyl->AXIS)), ff(cyl->center_bot_cap));
  real pd = len(pv) + r;
  if (pd > (real)cyl->radius) {
    c.normal = mk(-pv.x, -pv.y, -pv.z);
    c.normal = mulv(c.normal, (real)1.0 / len(c.normal));
    c.contact_point = sub(p, mulv(c.normal, r));
    c.dis = r_fabs(pd - (real)cyl->radius);
    c.is_collision = 1;
  }
  return c;
}

/* Drum/lifter surface velocity: cross((0,0,-MillRotVel), cp - (R,R,0)),
 * DEM_Kernels_Compute.cuh:377-380, 457-460 */
static v3 drum_velocity(const dem_oracle* o, v3 cp) {
  real R = (real)o->w[0].cyl_geo.radius;
  return cross(mk(0, 0, -(real)o->si.MillRotVel), sub(cp, mk(R, R, 0)));
}

/* WorldObject_InteractionParticle, DEM_Kernels_Compute.cuh:254-610 (spheres):
 * planar faces accumulate, the cylinder and its caps overwrite the force. */
static void world_forces(dem_oracle* o, int i, v3* fw_out, v3* tw_out) {
  const POBJ* P = &o->p[o->type[i]];
  v3 p = o->pos[i], v = o->vel[i], w = o->avel[i];
  const real r = o->rad[i], mass = o->mass[i];
  v3 fw = Z3, tw = Z3;
  for (int k = 0; k < o->num_wobj; ++k) {
    const WOBJ* W = &o->w[k];
    if (W->surface_type == plane) {
      for (int s = 0; s < W->num_surfaces; ++s) {
        coll_t c;
        if (W->surfaces[s].area == -1.0f)
          c = sphere_plane(p, r, ff(W->surfaces[s].normal), ff(W->surfaces[s].centroid));
        else
          c = sphere_surface(p, r, &W->surfaces[s], W->vertex);
        if (!c.is_collision) continue;
        forces_t F;
        if (o->si.Rotating_WObject && o->cyl_rot)
          F = law_moving_surface(o, c.normal, c.dis, sub(c.contact_point, p), w, P, v,
                                 drum_velocity(o, c.contact_point), mass);
        else
          F = law_static_surface(o, v, c.normal, c.dis, sub(c.contact_point, p), w, P, mass);
        fw = add(fw, F.trans);
        if (o->si.Rotation) tw = add(tw, F.torque);
      }
    } else if (W->surface_type == cylinder) {
      const Macro_Cylinder* cyl = &W->cyl_geo;
      coll_t c = sphere_cylinder(p, r, cyl);
      if (c.is_collision) {
        forces_t F;
        if (o->cyl_rot)
          F = law_moving_surface(o, c.normal, c.dis, sub(c.contact_point, p), w, P, v,
                                 drum_velocity(o, c.contact_point), mass);
        else
          F = law_static_surface(o, v, c.normal, c.dis, sub(c.contact_point, p), w, P, mass);
        fw = F.trans;
        if (o->si.Rotation) tw = add(tw, F.torque);
      }
      if (cyl->has_top_cap) {
        c = sphere_plane(p, r, ff(cyl->normal_top_cap), ff(cyl->center_top_cap));
        if (c.is_collision) {
          forces_t F = law_end_plate(v, c.normal, c.dis, P);
          fw = F.trans;
          if (o->si.Rotation) tw = add(tw, F.torque);
        }
      }
      if (cyl->has_bot_cap) {
        c = sphere_plane(p, r, ff(cyl->normal_bot_cap), ff(cyl->center_bot_cap));
        if (c.is_collision) {
          forces_t F = law_end_plate(v, c.normal, c.dis, P);
          fw = F.trans;
          if (o->si.Rotation) tw = add(tw, F.torque);
        }
      }
    }
  }
  *fw_out = fw;
  *tw_out = o->si.Rotation ? tw : Z3;
}

/* Collision_Detection_Sphere_DObject, Collision_Detection_Spheres.cuh:108-225 */
static coll_t sphere_dobject(const DOBJ* D, v3 p, real r, int hist_type) {
  coll_t c;
  c.is_collision = 0;
  c.colltype = 0;
  c.dis = 0;
  if (hist_type != 2) {
    for (int j = 0; j < D->num_faces; ++j) {
      const Surface* s = &D->faces[j];
      v3 n = ff(s->normal);
      v3 pt = sub(p, smul(r, n));
      c.dis = dot(n, sub(pt, ff(s->centroid)));
      if (c.dis < 0 && c.dis > -r * (real)0.5) {
        c.dis = r_fabs(c.dis);
        v3 q = add(pt, mulv(n, c.dis));
        if (point_on_surface(s->num_vertex, D->vertex, s->vertex_Order, q, (real)s->area, (real)s->Tol)) {
          c.is_collision = 1;
          c.contact_point = pt;
          c.normal = n;
          c.colltype = 1;
          return c;
        }
      }
    }
  }
  for (int e = 0; e < D->num_edges; ++e) {
    v3 pt0 = ff(D->vertex[D->edge[e].point_vindex[0]]);
    v3 dir = sub(ff(D->vertex[D->edge[e].point_vindex[1]]), pt0);
    v3 edir = divs(dir, len(dir));
    v3 vpc = sub(p, pt0);
    real dvec = dot(edir, vpc);
    if (dvec > 0) {
      v3 p2 = add(pt0, smul(dvec, edir));
      v3 d2 = sub(p, p2);
      real d = len(d2);
      if (d < r) {
        c.dis = r_fabs(d - r);
        if (c.dis < r) {
          c.normal = d2;
          c.normal = mulv(c.normal, (real)1.0 / len(c.normal));
          c.contact_point = Z3;
          c.colltype = 2;
          c.is_collision = 1;
          return c;
        }
      }
    }
  }
  return c;
}

/* VolumeObject_InteractionParticle, DEM_Kernels_Compute.cuh:12-246 (spheres):
 * bounding-cylinder test, faces then edges, first contact only. */
static void volume_forces(dem_oracle* o, int i, v3* fl_out, v3* tl_out) {
  const POBJ* P = &o->p[o->type[i]];
  v3 p = o->pos[i], v = o->vel[i], w = o->avel[i];
  const real r = o->rad[i], mass = o->mass[i];
  v3 fl = Z3, tl = Z3;
  int colltype = 0;
  int hist = o->lift_type[i];
  const DOBJ* D0 = &o->d[0];
  int outer = D0->is_translating || !o->si.isMillSim || o->si.Rotating_WObject;
  if (!outer) {
    v3 q = sub(mk(p.x, p.y, 0), ff(o->si.cent));
    outer = len(q) > ((real)o->si.DObject_CylinderBoundR - (real)2.0 * r);
  }
  if (outer) {
    for (int k = 0; k < o->n_d; ++k) {
      const DOBJ* D = &o->d[k];
      v3 bv = vmul(sub(p, ff(D->COM)), ff(D->Axis));
      if (!(len(bv) < ((real)D->boundR + r))) continue;
      coll_t c = sphere_dobject(D, p, r, hist);
      colltype = c.colltype;
      if (c.is_collision) {
        if (c.colltype == 2) c.contact_point = p;
        v3 vobj = Z3;
        if (D->is_attached_DWorld) vobj = drum_velocity(o, c.contact_point);
        else if (D->is_translating) vobj = ff(D->velocity);
        forces_t F = law_volume_object(o, c.normal, c.dis, sub(c.contact_point, p), w, P, v, vobj, mass);
        fl = add(fl, F.trans);
        if (o->si.Rotation) tl = add(tl, F.torque);
        break;
      }
    }
  }
  o->lift_type[i] = colltype;
  *fl_out = fl;
  *tl_out = tl;
}

/* ------------------------------------------------------------- integrate */
/* Integrate_Euler_NonSymmetry, Integration.cuh:6-184 (spheres, no quaternion) */
static void integrate(dem_oracle* o, int i) {
  const real dt = (real)o->si.InitalDelta_t;
  const real mass = o->mass[i];
  v3 acc = add(o->f_w[i], o->f_pp[i]);
  if (o->n_d > 0) acc = add(acc, o->f_l[i]);
  acc = mulv(acc, (real)1.0 / mass);
  o->vel[i] = add(o->vel[i], mulv(acc, dt));
  o->pos[i] = add(o->pos[i], mulv(o->vel[i], dt));
  if (o->si.Mode2D) o->vel[i].z = 0;
  v3 fl = add(o->t_pp[i], o->t_w[i]);
  if (o->n_d > 0) fl = add(fl, o->t_l[i]);
  if (o->si.Rotation) {
    if (dot(fl, fl) > 0) {
      v3 aa = smul(o->iinv[i], fl);
      o->avel[i] = add(o->avel[i], mulv(aa, dt));
      o->avel[i] = sub(o->avel[i], mulv(o->avel[i], (real)o->si.Roll_Res));
    }
    if (o->si.Mode2D) { o->avel[i].x = 0; o->avel[i].y = 0; }
  }
  if (!(isfinite((double)o->pos[i].x) && isfinite((double)o->pos[i].y) &&
        isfinite((double)o->pos[i].z)))
    o->status |= ST_NONFINITE;
}

/* --------------------------------------------------------------- one step */
static void step_once(dem_oracle* o) {
  const int n = o->n_cur;
  /* 1. hash (Kernel_SpatialDecomp_CalcPHash, BroadPhase.cuh:75-100) */
  for (int i = 0; i < n; ++i) {
    int g[3];
    grid_pos(o, o->pos[i], g);
    o->key[i] = grid_hash(o, g);
    o->idx[i] = i;
  }
  /* 2./3./4. sort and reorder */
  stable_sort(o, n);
  reorder(o, n);
  /* 5. drop killed particles: they carry the largest keys, DeviceInterface.cu:2062-2091 */
  if (o->num_dead > 0) {
    o->n_cur -= o->num_dead;
    o->num_dead = 0;
  }
  const int m = o->n_cur;
  /* 6. cell table (Kernel_SpatialDecomp_BinData, BroadPhase.cuh:279-325) */
  memset(o->cstart, 0xff, o->ncell * 4);
  memset(o->cend, 0xff, o->ncell * 4);
  for (int i = 0; i < m; ++i) {
    uint32_t h = o->key[i];
    if (h >= o->ncell) { o->status |= ST_OUT_OF_GRID; continue; }
    if (i == 0 || o->key[i - 1] != h) o->cstart[h] = (uint32_t)i;
    if (i == m - 1 || o->key[i + 1] != h) o->cend[h] = (uint32_t)i + 1;
  }
  for (int i = 0; i < m; ++i) {
    int g[3];
    grid_pos(o, o->pos[i], g);
    const int3 nc = o->si.num_NNCells;
    if (o->pid[i] > -1 && (g[0] < 0 || g[1] < 0 || g[2] < 0 || g[0] >= nc.x || g[1] >= nc.y || g[2] >= nc.z))
      o->status |= ST_OUT_OF_GRID;
  }
  /* 7. contact list */
  build_list(o, m);
  const int cap = o->law.max_nbr;
  /* 8. particle-particle forces (Kernel_ParticleInteraction_Spheres_NonSymmetry,
   *    DEM_Kernels_Compute.cuh:620-729) */
  for (int i = 0; i < m; ++i) {
    if (o->pid[i] <= -1) continue;
    const unsigned ta = o->type[i];
    v3 va = o->vel[i], pa = o->pos[i], wa = o->avel[i];
    const real ma = o->mass[i], ra = o->rad[i];
    v3 f = mulv(ff(o->si.Force_Field), ma);
    v3 fl = Z3;
    for (unsigned k = 0; k < o->nn[i]; ++k) {
      int j = (int)o->nlist[(size_t)i * cap + k];
      const unsigned tb = o->type[j];
      v3 pb = o->pos[j], vb = o->vel[j], wb = o->avel[j];
      const real rb = o->rad[j], mb = o->mass[j];
      v3 rel = sub(pa, pb);
      v3 rvel = sub(va, vb);
      real sep = len(rel) - (ra + rb);
      if (!(sep < 0)) continue; /* skin candidates that do not touch */
      v3 nrm = divs(rel, len(rel));
      real dis = r_fabs(len(rel) - (ra + rb)) + (real)0.000010f;
      forces_t F = law_pp_ref(o, rvel, nrm, dis, mulv(smul((real)-1.0, nrm), ra), mulv(nrm, rb),
                              wa, wb, &o->p[ta].PP[tb], va, vb, ma, mb);
      f = add(f, F.trans);
      fl = add(fl, F.torque);
    }
    o->f_pp[i] = f;
    o->t_pp[i] = o->si.Rotation ? fl : Z3;
  }
  /* 9. volume objects */
  if (o->n_d > 0)
    for (int i = 0; i < m; ++i)
      if (o->pid[i] > -1) volume_forces(o, i, &o->f_l[i], &o->t_l[i]);
  /* 10. world objects */
  for (int i = 0; i < m; ++i)
    if (o->pid[i] > -1) world_forces(o, i, &o->f_w[i], &o->t_w[i]);
  /* 11. integrate */
  for (int i = 0; i < m; ++i)
    if (o->pid[i] > -1) integrate(o, i);
  /* 13. silo kill every 1000 steps (DeviceInterface.cu:2463-2498); the
   * count is per check, not cumulative */
  if (o->si.Kill_Particles) {
    o->stepc++;
    if (o->stepc >= 1000) {
      int killed = 0;
      for (int i = 0; i < m; ++i) {
        if (o->pid[i] == -1) continue;
        int kill = 0;
        if (o->si.Rotating_WObject) {
          v3 q = o->pos[i];
          kill = q.z <= 41.0 || q.z >= 300 || q.y <= 50.0 || q.y >= 1500.0 || q.x <= 50.0 || q.x >= 1500.0;
        } else {
          kill = o->pos[i].y < (real)o->si.Silo_Kill_Height;
        }
        if (kill) {
          o->pos[i] = ff(o->si.max_size);
          o->pid[i] = -1;
          killed++;
        }
      }
      o->num_dead = killed;
      o->stepc = 0;
    }
  }
}

int dem_step(dem_oracle* o, int nsteps) {
  o->status = 0;
  for (int s = 0; s < nsteps; ++s) step_once(o);
  return o->status;
}

int dem_num_current(const dem_oracle* o) { return o->n_cur; }
int dem_status(const dem_oracle* o) { return o->status; }

void dem_get_state(const dem_oracle* o, double* pos3, double* vel3, double* avel3, unsigned* type,
                   int* pid) {
  for (int i = 0; i < o->n_max; ++i) {
    if (pos3) { pos3[3 * i] = o->pos[i].x; pos3[3 * i + 1] = o->pos[i].y; pos3[3 * i + 2] = o->pos[i].z; }
    if (vel3) { vel3[3 * i] = o->vel[i].x; vel3[3 * i + 1] = o->vel[i].y; vel3[3 * i + 2] = o->vel[i].z; }
    if (avel3) { avel3[3 * i] = o->avel[i].x; avel3[3 * i + 1] = o->avel[i].y; avel3[3 * i + 2] = o->avel[i].z; }
    if (type) type[i] = o->type[i];
    if (pid) pid[i] = o->pid[i];
  }
}

static void put(double* dst, const v3* src, int n) {
  if (!dst) return;
  for (int i = 0; i < n; ++i) { dst[3 * i] = src[i].x; dst[3 * i + 1] = src[i].y; dst[3 * i + 2] = src[i].z; }
}

void dem_get_forces(const dem_oracle* o, double* f_pp, double* t_pp, double* f_w, double* t_w,
                    double* f_l, double* t_l) {
  put(f_pp, o->f_pp, o->n_max); put(t_pp, o->t_pp, o->n_max);
  put(f_w, o->f_w, o->n_max); put(t_w, o->t_w, o->n_max);
  put(f_l, o->f_l, o->n_max); put(t_l, o->t_l, o->n_max);
}

void dem_get_nlist(const dem_oracle* o, unsigned* nn, unsigned* list) {
  const int cap = o->law.max_nbr;
  for (int i = 0; i < o->n_cur; ++i) {
    nn[i] = o->nn[i];
    for (int k = 0; k < cap; ++k) list[(size_t)i * cap + k] = k < (int)o->nn[i] ? o->nlist[(size_t)i * cap + k] : 0u;
  }
}

void dem_get_energy(const dem_oracle* o, double* e3) {
  e3[0] = o->e_pp * 1e-4;
  e3[1] = o->e_lift * 1e-4;
  e3[2] = o->e_surf * 1e-4;
}
