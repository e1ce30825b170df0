/*
 * ens_oracle.c -- CPU restatement of the ensemble path (include/blaze_ens.h):
 * system-prefixed cell keys, stable sort, Verlet list with tangential-history
 * carry-over, the linear / Hertz-Mindlin contact law with history, Coulomb
 * cap and rolling friction, plane / cylinder / triangle walls, symplectic
 * Euler.  Compiled twice: DEM_REAL=float follows the product's FP32
 * operation order (compile with -ffp-contract=off), DEM_REAL=double is the
 * FP64 oracle the FP32 error is stated against.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it as the checker; the product never does.
 *
 * The reference has no such laws (its law is Collision_Response.cuh:374-494),
 * so this restatement is the only pin of these results: parity unpinned vs
 * the reference.  The step structure follows the reference's step
 * (DeviceInterface.cu:1825-2513): hash, stable sort, reorder, cell table,
 * 27-cell search, per-particle force gather, symplectic Euler
 * (Integration.cuh:6-184).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/blaze_ens.h"

#ifndef DEM_REAL
#define DEM_REAL double
#endif
typedef DEM_REAL real;

#define IS_FLOAT (sizeof(real) == sizeof(float))
static real SQRT(real x) { return IS_FLOAT ? (real)sqrtf((float)x) : (real)sqrt((double)x); }
static real FLOOR(real x) { return IS_FLOAT ? (real)floorf((float)x) : (real)floor((double)x); }
static real IN(double x) { return IS_FLOAT ? (real)(float)x : (real)x; }

typedef struct { real x, y, z; } v3;
static v3 mk(real x, real y, real z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, real s) { return mk(a.x * s, a.y * s, a.z * s); }
static v3 smul(real s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static real dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static real len(v3 a) { return SQRT(dot(a, a)); }
static v3 cross(v3 a, v3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

enum { WSLOTS = 4 };
enum { ST_OVERFLOW = 1, ST_OUT_OF_GRID = 2, ST_NONFINITE = 4 };

typedef struct {
  v3 origin;
  real cell;
  int nc[3];
  uint32_t cell_off;
  v3 g;
  real dens43pi, kn, kt, beta2, estar, gstar, beta2h, mu, mu_w, mu_r;
  int wall0, nwall, tri0, ntri;
  /* turning drum (blaze_system.rot_*), csrc/ens_kernels.cu "drum turn" */
  v3 rot_o, rot_a;
  real rot_w, rot_cd, rot_sd;
  int rot;
} sysc;

typedef struct {
  int kind;
  int turning;   /* turns in place with its system's drum: its surface moves */
  real r;
  v3 a, b, c;
  double n64[3], e64[3][3];   /* triangle: unit normal, unit edges ab, ac, bc (double) */
} wallc;

/* Accurate overlaps (csrc/ens_kernels.cuh, "accurate overlaps"): formed in
 * double from the working-precision state, as the kernels do, then rounded
 * to the working precision once. */
static double dotd(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static real overlap_pair(real ra, real rb, v3 pa, v3 pb) {
  const double d[3] = {(double)pa.x - (double)pb.x, (double)pa.y - (double)pb.y,
                       (double)pa.z - (double)pb.z};
  return (real)(((double)ra + (double)rb) - sqrt(dotd(d, d)));
}
static real overlap_plane(real r, v3 n, real d, v3 p) {
  const double nn[3] = {n.x, n.y, n.z}, pp[3] = {p.x, p.y, p.z};
  return (real)(((double)r + (double)d) - dotd(nn, pp));
}
static void unit64(double x, double y, double z, double* u) {
  const double l = sqrt(x * x + y * y + z * z);
  u[0] = l > 0 ? x / l : 0.0;
  u[1] = l > 0 ? y / l : 0.0;
  u[2] = l > 0 ? z / l : 0.0;
}

typedef struct {
  v3 pos, vel, w;
  real r, path;       /* a polyhedron: r = its bounding radius; path kept per polyhedron */
  int sys, pid;
  int poly;           /* polyhedron id, -1 for a sphere */
  uint32_t wmask;
  real wh[WSLOTS][3];
  int wid[WSLOTS];
} part;

typedef struct ens_oracle ens_oracle;
struct ens_oracle {
  int law, n, nsys, nwalls, cap;
  real dt, skin;
  sysc* S;
  wallc* W;
  uint32_t ncell_tab;
  part* p;      /* current state, memory order */
  part* q;      /* scratch */
  /* two list copies: idx, cnt, mask, history */
  uint32_t* idx[2];
  uint32_t* cnt[2];
  uint32_t* mask[2];
  real* hist[2];    /* [k * n + i][3] */
  int epoch;
  int rebuild_req;
  uint32_t status;
  uint32_t* cstart;
  uint32_t* cend;
  v3* cap_f;
  v3* cap_t;
  int* sys_of;      /* system of each entry of the caller's arrays */
  real* rot_c;      /* per system: cosine and sine of the drum's turn so far */
  real* rot_s;
  struct tstep_* tape; /* recorded steps of the reverse sweep */
  int ntape;
  struct mixc_* mix;   /* polyhedra among the spheres (NULL: spheres only) */
  /* candidate triangles per cell (CSR over the global cell table), as the
     library bins them; with use_tri_lists 0 every triangle of the system is
     tested (the same contacts: the lists hold every triangle a particle
     centred in the cell can touch) */
  uint32_t* tri_off;
  uint32_t* tri_ids;
  int use_tri_lists;
};

static void constants(sysc* d, const blaze_system* s, uint32_t off, float dt) {
  const double pi = 3.14159265358979323846;
  const double e = s->restitution;
  const double le = log(e);
  const double beta = -le / sqrt(le * le + pi * pi);
  const double E = s->youngs, nu = s->poisson;
  d->origin = mk(s->origin[0], s->origin[1], s->origin[2]);
  d->cell = s->cell;
  d->nc[0] = s->ncells[0]; d->nc[1] = s->ncells[1]; d->nc[2] = s->ncells[2];
  d->cell_off = off;
  d->g = mk(s->gravity[0], s->gravity[1], s->gravity[2]);
  /* the FP32 build rounds each constant once, as the product's host code does */
  d->dens43pi = (real)((double)s->density * 4.0 / 3.0 * pi);
  d->kn = s->kn;
  d->kt = (real)((double)s->kn * (double)s->kt_ratio);
  d->beta2 = (real)(2.0 * beta);
  d->estar = (real)(E / (2.0 * (1.0 - nu * nu)));
  d->gstar = (real)(E / (4.0 * (2.0 - nu) * (1.0 + nu)));
  d->beta2h = (real)(2.0 * sqrt(5.0 / 6.0) * beta);
  d->mu = s->mu; d->mu_w = s->mu_wall; d->mu_r = s->mu_roll;
  d->wall0 = s->wall0; d->nwall = s->nwalls; d->tri0 = s->tri0; d->ntri = s->ntris;
  d->rot_o = mk(s->rot_point[0], s->rot_point[1], s->rot_point[2]);
  d->rot_a = mk(s->rot_axis[0], s->rot_axis[1], s->rot_axis[2]);
  d->rot_w = s->rot_omega;
  d->rot = s->rot_omega != 0.0f;
  {
    const float ang = s->rot_omega * dt;   /* single-precision cosine and sine, as the host */
    d->rot_cd = (real)cosf(ang);
    d->rot_sd = (real)sinf(ang);
  }
}

/* v turned by the angle with cosine c and sine s about the unit axis a:
 * v c + (a x v) s + a (a . v) (1 - c), in the kernels' order */
static v3 rot_about(v3 a, real c, real s, v3 v) {
  const v3 axv = cross(a, v);
  const real av = dot(a, v);
  return add(add(mul(v, c), mul(axv, s)), mul(a, av * ((real)1.0 - c)));
}

typedef struct { uint32_t cell, tri; } ctpair;
static int ctpair_cmp(const void* a, const void* b) {
  const ctpair* x = (const ctpair*)a;
  const ctpair* y = (const ctpair*)b;
  if (x->cell != y->cell) return x->cell < y->cell ? -1 : 1;
  return x->tri < y->tri ? -1 : (x->tri > y->tri);
}

/* Candidate triangles per cell (csrc/ens_capi.cu, build_tri_lists): every
 * cell whose box meets the triangle's bounding box grown by half a cell,
 * in ascending triangle order. */
static void build_tri_lists(ens_oracle* o, const blaze_system* sys) {
  size_t np = 0, cap = 1024;
  ctpair* pr = (ctpair*)malloc(sizeof(ctpair) * cap);
  for (int s = 0; s < o->nsys; ++s) {
    const blaze_system* S = &sys[s];
    const double cell = (double)S->cell;
    const double margin = 0.5 * cell + 1e-4 * cell;
    for (int t = S->tri0; t < S->tri0 + S->ntris; ++t) {
      const wallc* W = &o->W[t];
      const v3 v[3] = {W->a, W->b, W->c};
      int lo[3], hi[3];
      for (int c = 0; c < 3; ++c) {
        double mn = 1e300, mx = -1e300;
        for (int k = 0; k < 3; ++k) {
          const double x = (double)(float)(c == 0 ? v[k].x : (c == 1 ? v[k].y : v[k].z));
          if (x < mn) mn = x;
          if (x > mx) mx = x;
        }
        const double og = (double)S->origin[c];
        const int ncs = S->ncells[c];
        const int l = (int)floor((mn - margin - og) / cell), h = (int)floor((mx + margin - og) / cell);
        lo[c] = l > 0 ? l : 0;
        hi[c] = h < ncs - 1 ? h : ncs - 1;
      }
      for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
          for (int x = lo[0]; x <= hi[0]; ++x) {
            if (np == cap) { cap *= 2; pr = (ctpair*)realloc(pr, sizeof(ctpair) * cap); }
            pr[np].cell = o->S[s].cell_off + (uint32_t)(x + S->ncells[0] * (y + S->ncells[1] * z));
            pr[np].tri = (uint32_t)t;
            ++np;
          }
    }
  }
  qsort(pr, np, sizeof(ctpair), ctpair_cmp);
  o->tri_off = (uint32_t*)calloc((size_t)o->ncell_tab + 1, sizeof(uint32_t));
  o->tri_ids = (uint32_t*)malloc(sizeof(uint32_t) * (np ? np : 1));
  for (size_t k = 0; k < np; ++k) {
    o->tri_off[pr[k].cell + 1]++;
    o->tri_ids[k] = pr[k].tri;
  }
  for (uint32_t c = 0; c < o->ncell_tab; ++c) o->tri_off[c + 1] += o->tri_off[c];
  free(pr);
}

/* Test infrastructure switch: 0 tests every triangle of a system (the
 * restatement's first form), 1 the candidates of the particle's cell. */
void ens_use_tri_lists(ens_oracle* o, int on) { o->use_tri_lists = on; }

ens_oracle* ens_create(const blaze_system* sys, int nsys, const blaze_wall* walls, int nwalls,
                       int law, double dt, double skin, int max_nbr) {
  ens_oracle* o = (ens_oracle*)calloc(1, sizeof(ens_oracle));
  o->law = law; o->nsys = nsys; o->nwalls = nwalls; o->cap = max_nbr;
  o->dt = (real)(float)dt;
  o->skin = (real)(float)skin;
  o->S = (sysc*)calloc(nsys, sizeof(sysc));
  uint32_t off = 0;
  int n = 0;
  for (int s = 0; s < nsys; ++s) {
    constants(&o->S[s], &sys[s], off, (float)dt);
    off += (uint32_t)sys[s].ncells[0] * sys[s].ncells[1] * sys[s].ncells[2];
    n += sys[s].n;
  }
  o->ncell_tab = off;
  o->n = n;
  o->W = (wallc*)calloc(nwalls > 0 ? nwalls : 1, sizeof(wallc));
  for (int w = 0; w < nwalls; ++w) {
    const float* p = walls[w].p;
    wallc* d = &o->W[w];
    d->kind = walls[w].kind;
    if (d->kind == BLAZE_WALL_PLANE) { d->a = mk(p[0], p[1], p[2]); d->r = p[3]; }
    else if (d->kind == BLAZE_WALL_TRIANGLE) {
      d->a = mk(p[0], p[1], p[2]); d->b = mk(p[3], p[4], p[5]); d->c = mk(p[6], p[7], p[8]);
      const double ab[3] = {(double)p[3] - p[0], (double)p[4] - p[1], (double)p[5] - p[2]};
      const double ac[3] = {(double)p[6] - p[0], (double)p[7] - p[1], (double)p[8] - p[2]};
      const double bc[3] = {(double)p[6] - p[3], (double)p[7] - p[4], (double)p[8] - p[5]};
      unit64(ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
             ab[0] * ac[1] - ab[1] * ac[0], d->n64);
      unit64(ab[0], ab[1], ab[2], d->e64[0]);
      unit64(ac[0], ac[1], ac[2], d->e64[1]);
      unit64(bc[0], bc[1], bc[2], d->e64[2]);
    } else { d->a = mk(p[0], p[1], p[2]); d->b = mk(p[3], p[4], p[5]); d->r = p[6]; }
  }
  /* walls that turn in place with a drum (csrc/ens_capi.cu, create_impl) */
  for (int s = 0; s < nsys; ++s) {
    const blaze_system* y = &sys[s];
    if (y->rot_omega == 0.0f) continue;
    const double ax = y->rot_axis[0], ay = y->rot_axis[1], az = y->rot_axis[2];
    for (int w = y->wall0; w < y->wall0 + y->nwalls; ++w) {
      wallc* W = &o->W[w];
      const double a[3] = {(float)W->a.x, (float)W->a.y, (float)W->a.z};
      const double b[3] = {(float)W->b.x, (float)W->b.y, (float)W->b.z};
      if (W->kind == BLAZE_WALL_PLANE) {
        W->turning = fabs(fabs(a[0] * ax + a[1] * ay + a[2] * az) - 1.0) < 1e-6;
      } else if (W->kind == BLAZE_WALL_CYLINDER) {
        const double par = fabs(b[0] * ax + b[1] * ay + b[2] * az);
        const double d[3] = {a[0] - y->rot_point[0], a[1] - y->rot_point[1], a[2] - y->rot_point[2]};
        const double dd = d[0] * ax + d[1] * ay + d[2] * az;
        const double q = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] - dd * dd;
        W->turning = fabs(par - 1.0) < 1e-6 && sqrt(q > 0 ? q : 0) < 1e-4;
      }
    }
  }
  o->p = (part*)calloc(n, sizeof(part));
  o->q = (part*)calloc(n, sizeof(part));
  for (int c = 0; c < 2; ++c) {
    o->idx[c] = (uint32_t*)calloc((size_t)n * max_nbr, sizeof(uint32_t));
    o->cnt[c] = (uint32_t*)calloc(n, sizeof(uint32_t));
    o->mask[c] = (uint32_t*)calloc(n, sizeof(uint32_t));
    o->hist[c] = (real*)calloc((size_t)n * max_nbr * 3, sizeof(real));
  }
  o->cstart = (uint32_t*)malloc(sizeof(uint32_t) * (o->ncell_tab ? o->ncell_tab : 1));
  o->cend = (uint32_t*)malloc(sizeof(uint32_t) * (o->ncell_tab ? o->ncell_tab : 1));
  o->cap_f = (v3*)calloc(n, sizeof(v3));
  o->cap_t = (v3*)calloc(n, sizeof(v3));
  o->sys_of = (int*)calloc(n, sizeof(int));
  o->rot_c = (real*)calloc(nsys, sizeof(real));
  o->rot_s = (real*)calloc(nsys, sizeof(real));
  for (int s = 0; s < nsys; ++s) o->rot_c[s] = 1;
  int k = 0;
  for (int s = 0; s < nsys; ++s)
    for (int m = 0; m < sys[s].n; ++m) o->sys_of[k++] = s;
  build_tri_lists(o, sys);
  o->use_tri_lists = 1;
  return o;
}

static void free_tape(ens_oracle* o);
static void free_mix(ens_oracle* o);
void ens_destroy(ens_oracle* o) {
  if (!o) return;
  free_tape(o);
  free_mix(o);
  free(o->S); free(o->W); free(o->p); free(o->q);
  for (int c = 0; c < 2; ++c) { free(o->idx[c]); free(o->cnt[c]); free(o->mask[c]); free(o->hist[c]); }
  free(o->cstart); free(o->cend); free(o->cap_f); free(o->cap_t); free(o->sys_of);
  free(o->rot_c); free(o->rot_s); free(o->tri_off); free(o->tri_ids);
  free(o);
}

/* The five law constants of system s that the reverse sweep differentiates
 * (kn, kt, 2 beta, mu, mu_wall), read or set directly in working precision
 * (finite differences in FP64 go through these). */
void ens_get_constants(const ens_oracle* o, int s, double* c5) {
  const sysc* S = &o->S[s];
  c5[0] = S->kn; c5[1] = S->kt; c5[2] = S->beta2; c5[3] = S->mu; c5[4] = S->mu_w;
}
void ens_set_constants(ens_oracle* o, int s, const double* c5) {
  sysc* S = &o->S[s];
  S->kn = (real)c5[0]; S->kt = (real)c5[1]; S->beta2 = (real)c5[2]; S->mu = (real)c5[3];
  S->mu_w = (real)c5[4];
}

int ens_set_params(ens_oracle* o, const blaze_system* sys) {
  for (int s = 0; s < o->nsys; ++s) constants(&o->S[s], &sys[s], o->S[s].cell_off, (float)o->dt);
  return 0;
}

void ens_set_state(ens_oracle* o, const double* pos3, const double* rad, const double* vel3,
                   const double* avel3) {
  for (int i = 0; i < o->n; ++i) {
    part* a = &o->p[i];
    memset(a, 0, sizeof(*a));
    a->sys = o->sys_of[i];
    /* the FP32 build takes the inputs as the product does (rounded to
       float); the FP64 build keeps them exact, so finite differences of
       size 1e-6 are resolved */
    a->pos = mk(IN(pos3[3 * i]), IN(pos3[3 * i + 1]), IN(pos3[3 * i + 2]));
    a->r = (real)(float)rad[i];
    if (vel3) a->vel = mk(IN(vel3[3 * i]), IN(vel3[3 * i + 1]), IN(vel3[3 * i + 2]));
    if (avel3) a->w = mk(IN(avel3[3 * i]), IN(avel3[3 * i + 1]), IN(avel3[3 * i + 2]));
    a->pid = i;
    a->poly = -1;
    for (int q = 0; q < WSLOTS; ++q) a->wid[q] = -1;
  }
  free_mix(o);   /* spheres only again */
  for (int c = 0; c < 2; ++c) {
    memset(o->cnt[c], 0, sizeof(uint32_t) * o->n);
    memset(o->mask[c], 0, sizeof(uint32_t) * o->n);
  }
  o->rebuild_req = 1;
  o->status = 0;
  for (int s = 0; s < o->nsys; ++s) { o->rot_c[s] = 1; o->rot_s[s] = 0; }
}

static int cell_of(const sysc* S, v3 p, int c[3]) {
  c[0] = (int)FLOOR((p.x - S->origin.x) / S->cell);
  c[1] = (int)FLOOR((p.y - S->origin.y) / S->cell);
  c[2] = (int)FLOOR((p.z - S->origin.z) / S->cell);
  return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < S->nc[0] && c[1] < S->nc[1] && c[2] < S->nc[2];
}
static uint32_t key_of(const sysc* S, const int c[3]) {
  return S->cell_off + (uint32_t)(c[0] + S->nc[0] * (c[1] + S->nc[1] * c[2]));
}

typedef struct { uint32_t key; int idx; } kv;
static int kv_cmp(const void* a, const void* b) {
  const kv* x = (const kv*)a;
  const kv* y = (const kv*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* Re-sort + new list.  When `perm_out` / `src_out` are given they receive,
 * for the tape of the reverse sweep, the old index of each new position and
 * the old slot each new slot's history came from (-1: none). */
static void rebuild_rec(ens_oracle* o, int* perm_out, int* src_out);
static void rebuild(ens_oracle* o) { rebuild_rec(o, NULL, NULL); }
static void mix_rebuild_lists(ens_oracle* o);
static void rebuild_rec(ens_oracle* o, int* perm_out, int* src_out) {
  const int n = o->n, cap = o->cap;
  const int e = o->epoch & 1;
  kv* ks = (kv*)malloc(sizeof(kv) * n);
  for (int i = 0; i < n; ++i) {
    const sysc* S = &o->S[o->p[i].sys];
    int c[3];
    if (cell_of(S, o->p[i].pos, c)) ks[i].key = key_of(S, c);
    else { ks[i].key = o->ncell_tab; o->status |= ST_OUT_OF_GRID; }
    ks[i].idx = i;
  }
  qsort(ks, n, sizeof(kv), kv_cmp);   /* (key, index): the stable order */
  for (uint32_t h = 0; h < o->ncell_tab; ++h) o->cstart[h] = 0xffffffffu;
  for (int i = 0; i < n; ++i) {
    o->q[i] = o->p[ks[i].idx];
    o->q[i].path = 0;
    const uint32_t k = ks[i].key;
    if (k < o->ncell_tab) {
      if (i == 0 || ks[i - 1].key != k) o->cstart[k] = (uint32_t)i;
      if (i == n - 1 || ks[i + 1].key != k) o->cend[k] = (uint32_t)i + 1u;
    }
  }
  /* neighbour list of the new order, history carried by partner pid */
  uint32_t *Io = o->idx[e], *In = o->idx[e ^ 1];
  uint32_t *Co = o->cnt[e], *Cn = o->cnt[e ^ 1];
  uint32_t *Mo = o->mask[e], *Mn = o->mask[e ^ 1];
  real *Ho = o->hist[e], *Hn = o->hist[e ^ 1];
  for (int i = 0; i < n; ++i) {
    const part* a = &o->q[i];
    if (a->poly >= 0) {   /* a polyhedron: its own list (mix_rebuild_lists) */
      Cn[i] = 0;
      Mn[i] = 0;
      continue;
    }
    const sysc* S = &o->S[a->sys];
    const int io = ks[i].idx;
    const uint32_t cnt_o = Co[io], mask_o = Mo[io];
    uint32_t cnt = 0, mask = 0;
    int c[3];
    if (cell_of(S, a->pos, c)) {
      const int x0 = c[0] > 0 ? c[0] - 1 : 0, x1 = c[0] < S->nc[0] - 1 ? c[0] + 1 : c[0];
      const int y0 = c[1] > 0 ? c[1] - 1 : 0, y1 = c[1] < S->nc[1] - 1 ? c[1] + 1 : c[1];
      const int z0 = c[2] > 0 ? c[2] - 1 : 0, z1 = c[2] < S->nc[2] - 1 ? c[2] + 1 : c[2];
      for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
          for (int x = x0; x <= x1; ++x) {
            const uint32_t h = S->cell_off + (uint32_t)(S->nc[0] * (y + S->nc[1] * z)) + (uint32_t)x;
            const uint32_t s0 = o->cstart[h];
            if (s0 == 0xffffffffu) continue;
            for (uint32_t j = s0; j < o->cend[h]; ++j) {
              if ((int)j == i) continue;
              const part* b = &o->q[j];
              const v3 rel = sub(a->pos, b->pos);
              const real lim = (a->r + b->r) + o->skin;
              if (!(dot(rel, rel) < lim * lim)) continue;
              if (cnt < (uint32_t)cap) {
                In[(size_t)cnt * n + i] = j;
                if (src_out) src_out[(size_t)cnt * n + i] = -1;
                for (uint32_t ko = 0; ko < cnt_o && ko < 32; ++ko) {
                  if (!((mask_o >> ko) & 1u)) continue;
                  const size_t so = (size_t)ko * n + io;
                  if (o->p[Io[so]].pid == b->pid) {
                    const size_t sn = (size_t)cnt * n + i;
                    Hn[3 * sn] = Ho[3 * so]; Hn[3 * sn + 1] = Ho[3 * so + 1]; Hn[3 * sn + 2] = Ho[3 * so + 2];
                    if (src_out) src_out[sn] = (int)ko;
                    mask |= 1u << cnt;
                    break;
                  }
                }
              } else {
                o->status |= ST_OVERFLOW;
              }
              ++cnt;
            }
          }
    } else {
      o->status |= ST_OUT_OF_GRID;
    }
    Cn[i] = cnt < (uint32_t)cap ? cnt : (uint32_t)cap;
    Mn[i] = mask;
  }
  if (perm_out)
    for (int i = 0; i < n; ++i) perm_out[i] = ks[i].idx;
  if (o->mix) mix_rebuild_lists(o);
  part* t = o->p; o->p = o->q; o->q = t;
  o->epoch += 1;
  free(ks);
}

static void contact_law(const ens_oracle* o, const sysc* S, real mu, v3 n, real delta, real rs,
                        real ms, v3 vrel, v3 vct, v3 wrel, real arm, v3* xi, v3* F, v3* T) {
  const real vn = dot(vrel, n);
  real kn_e, cn, kt_e, ct;
  if (o->law == BLAZE_LAW_LINEAR) {
    kn_e = S->kn;
    kt_e = S->kt;
    cn = S->beta2 * SQRT(ms * S->kn);
    ct = S->beta2 * SQRT(ms * S->kt);
  } else {
    const real sq = SQRT(rs * delta);
    const real sn = ((real)2.0 * S->estar) * sq;
    kn_e = (real)(2.0 / 3.0) * sn;
    kt_e = ((real)8.0 * S->gstar) * sq;
    cn = S->beta2h * SQRT(sn * ms);
    ct = S->beta2h * SQRT(kt_e * ms);
  }
  const real fn = kn_e * delta - cn * vn;
  const real fc = fn > 0 ? fn : 0;
  const v3 vt = sub(vct, smul(dot(vct, n), n));
  v3 x = *xi;
  const real xn = dot(x, n);
  if (xn != 0) {
    const real m0 = dot(x, x);
    x = sub(x, smul(xn, n));
    const real m1 = dot(x, x);
    if (m1 > 0) x = mul(x, SQRT(m0 / m1));
  }
  x = add(x, mul(vt, o->dt));
  v3 ft = sub(mul(x, -kt_e), mul(vt, ct));
  const real capf = mu * fc;
  const real f2 = dot(ft, ft);
  if (f2 > capf * capf) {
    const real s = capf / SQRT(f2);
    ft = mul(ft, s);
    x = mul(add(ft, mul(vt, ct)), (real)-1.0 / kt_e);
  }
  *xi = x;
  *F = add(mul(n, fn), ft);
  *T = cross(mul(n, -arm), *F);
  if (S->mu_r > 0) {
    const real w2 = dot(wrel, wrel);
    if (w2 > 0) *T = add(*T, mul(wrel, -((S->mu_r * fc) * rs) / SQRT(w2)));
  }
}

static v3 closest_tri(v3 p, v3 a, v3 b, v3 c, int* region, int* feat) {
  const v3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const real d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) { *region = 2; *feat = 0; return a; }
  const v3 bp = sub(p, b);
  const real d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) { *region = 2; *feat = 1; return b; }
  const real vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    *region = 1; *feat = 0;
    return add(a, mul(ab, d1 / (d1 - d3)));
  }
  const v3 cp = sub(p, c);
  const real d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) { *region = 2; *feat = 2; return c; }
  const real vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    *region = 1; *feat = 1;
    return add(a, mul(ac, d2 / (d2 - d6)));
  }
  const real va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    *region = 1; *feat = 2;
    return add(b, mul(sub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
  }
  const real den = (real)1.0 / ((va + vb) + vc);
  *region = 0; *feat = 0;
  return add(add(a, mul(ab, vb * den)), mul(ac, vc * den));
}

static int wall_touch(const wallc* W, v3 p, real r, v3* n, real* delta, int* region) {
  *region = 0;
  /* the kernels' conservative pre-test (a contact is never rejected by it) */
  const real mag = (real)fabs((double)p.x) + (real)fabs((double)p.y) + (real)fabs((double)p.z) +
                   (real)fabs((double)W->r);
  if (W->kind == BLAZE_WALL_PLANE) {
    if (!(dot(W->a, p) - W->r < r + (real)1e-6 * mag)) return 0;
    *delta = overlap_plane(r, W->a, W->r, p);
    if (!(*delta > 0)) return 0;
    *n = W->a;
    return 1;
  }
  if (W->kind == BLAZE_WALL_CYLINDER) {
    {
      const v3 v = sub(p, W->a);
      if (!(len(sub(v, smul(dot(v, W->b), W->b))) + r > W->r - (real)1e-6 * (mag + 2 * W->r)))
        return 0;
    }
    const double v[3] = {(double)p.x - (double)W->a.x, (double)p.y - (double)W->a.y,
                         (double)p.z - (double)W->a.z};
    const double b[3] = {W->b.x, W->b.y, W->b.z};
    const double vb = dotd(v, b);
    const double rad[3] = {v[0] - vb * b[0], v[1] - vb * b[1], v[2] - vb * b[2]};
    const double rho = sqrt(dotd(rad, rad));
    *delta = (real)(((double)r + rho) - (double)W->r);
    if (!(*delta > 0) || !(rho > 0)) return 0;
    const real rinv = (real)(-1.0 / rho);
    *n = mk((real)rad[0] * rinv, (real)rad[1] * rinv, (real)rad[2] * rinv);
    return 1;
  }
  int feat;
  const v3 q = closest_tri(p, W->a, W->b, W->c, region, &feat);
  const v3 d = sub(p, q);
  const real d2 = dot(d, d);
  if (!(d2 < r * r)) return 0;
  if (*region == 0) {
    const double pa[3] = {(double)p.x - (double)W->a.x, (double)p.y - (double)W->a.y,
                          (double)p.z - (double)W->a.z};
    const double s = dotd(pa, W->n64);
    *delta = (real)((double)r - fabs(s));
    if (!(*delta > 0) || !(s != 0.0)) return 0;
    const real sg = s < 0.0 ? (real)-1.0 : (real)1.0;
    *n = mk((real)W->n64[0] * sg, (real)W->n64[1] * sg, (real)W->n64[2] * sg);
    return 1;
  }
  const v3 v0 = *region == 2 ? (feat == 0 ? W->a : (feat == 1 ? W->b : W->c))
                             : (feat == 2 ? W->b : W->a);
  double pv[3] = {(double)p.x - (double)v0.x, (double)p.y - (double)v0.y,
                  (double)p.z - (double)v0.z};
  if (*region == 1) {
    const double* e = W->e64[feat];
    const double t = dotd(pv, e);
    pv[0] = pv[0] - t * e[0];
    pv[1] = pv[1] - t * e[1];
    pv[2] = pv[2] - t * e[2];
  }
  const double dist = sqrt(dotd(pv, pv));
  *delta = (real)((double)r - dist);
  if (!(*delta > 0) || !(dist > 0)) return 0;
  const real dinv = (real)(1.0 / dist);
  *n = mk((real)pv[0] * dinv, (real)pv[1] * dinv, (real)pv[2] * dinv);
  return 1;
}

typedef struct {
  const ens_oracle* o;
  const sysc* S;
  const part* a;
  real ma;
  v3 f, t;
  int nw;
  real nh[WSLOTS][3];
  int nid[WSLOTS];
  uint32_t st;
} wctx;

static void wall_contact(wctx* c, int id, v3 n, real delta, int moving) {
  const part* a = c->a;
  const sysc* S = c->S;
  v3 xi = mk(0, 0, 0);
  for (int q = 0; q < WSLOTS; ++q)
    if (((a->wmask >> q) & 1u) && a->wid[q] == id) xi = mk(a->wh[q][0], a->wh[q][1], a->wh[q][2]);
  const v3 vcpa = add(a->vel, cross(a->w, mul(n, -a->r)));
  v3 vr = a->vel, vc = vcpa, wr = a->w;
  if (moving) {
    /* the wall's velocity at the contact point, and its spin */
    const v3 vw = mul(cross(S->rot_a, sub(sub(a->pos, mul(n, a->r)), S->rot_o)), S->rot_w);
    vr = sub(a->vel, vw);
    vc = sub(vcpa, vw);
    wr = sub(a->w, mul(S->rot_a, S->rot_w));
  }
  v3 F, T;
  contact_law(c->o, c->S, c->S->mu_w, n, delta, a->r, c->ma, vr, vc, wr, a->r, &xi, &F, &T);
  c->f = add(c->f, F);
  c->t = add(c->t, T);
  if (c->nw < WSLOTS) {
    c->nh[c->nw][0] = xi.x; c->nh[c->nw][1] = xi.y; c->nh[c->nw][2] = xi.z;
    c->nid[c->nw] = id;
    c->nw++;
  } else {
    c->st |= ST_OVERFLOW;
  }
}

/* ============================================================ polyhedra
 * Convex polyhedra among the spheres of a system (csrc/mix_device.cuh,
 * csrc/mix_kernels.cu): the same shapes, narrow phases (FP64 from the
 * working-precision state), laws and integration, stepped one particle at a
 * time.  The polyhedron's own force sums its list slots in slot order, then
 * the planes in order, then the kept triangles in ascending order. */
enum { MIX_V = 16, MIX_F = 28, MIX_E = 42, MIX_SLOTS = 64, MIX_WSLOTS = 16 };

typedef struct {
  int nv, nf, ne;
  real mass, inertia[9], iinv[9];
  float rb;                  /* bounding radius, rounded up to float */
  double bv[MIX_V][3];       /* body vertices (the float inputs) */
  double bn[MIX_F][3];       /* body unit normals */
  int faces[MIX_F][3];
  int edges[MIX_E][4];       /* vertex i < j, faces f1 < f2 */
} mshape;

typedef struct mixc_ {
  int npoly, nshape;
  mshape* shapes;
  int* shape_of;             /* per polyhedron */
  real* quat;                /* per polyhedron: w x y z */
  real* path;
  int* pat;                  /* memory position */
  double* gv;                /* per polyhedron: MIX_V x 4 (offset from the centre) */
  double* gf;                /* per polyhedron: MIX_F x 4 (unit normal, offset h) */
  real* wh;                  /* per polyhedron: MIX_WSLOTS wall histories (xi) */
  int* wid;                  /* their wall ids */
  int* wn;                   /* slots in use */
  uint32_t* idx[2];          /* slot k of polyhedron p at k * npoly + p */
  uint32_t* cnt[2];
  uint64_t* mask[2];
  real* hist[2];
} mixc;

static void free_mix(ens_oracle* o) {
  mixc* m = o->mix;
  if (!m) return;
  free(m->shapes); free(m->shape_of); free(m->quat); free(m->path); free(m->pat);
  free(m->gv); free(m->gf); free(m->wh); free(m->wid); free(m->wn);
  for (int c = 0; c < 2; ++c) { free(m->idx[c]); free(m->cnt[c]); free(m->mask[c]); free(m->hist[c]); }
  free(m);
  o->mix = NULL;
}

static int edge_cmp(const void* a, const void* b) {
  const int* x = (const int*)a;
  const int* y = (const int*)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

/* Shape of a blaze_shape (csrc/ens_capi.cu, shape_setup): unit normals,
 * edges, and mass properties from the tetrahedra of the faces with the
 * origin, in FP64 in the same order of operations. */
static int mix_shape(const blaze_shape* s, mshape* o) {
  memset(o, 0, sizeof(*o));
  const int nv = s->nverts, nf = s->nfaces;
  if (nv < 4 || nv > MIX_V || nf != 2 * nv - 4 || !(s->density > 0.0f)) return -1;
  o->nv = nv;
  o->nf = nf;
  for (int k = 0; k < nv; ++k)
    for (int c = 0; c < 3; ++c) o->bv[k][c] = (double)s->verts[3 * k + c];
  for (int f = 0; f < nf; ++f) {
    const int a = s->faces[3 * f], b = s->faces[3 * f + 1], c = s->faces[3 * f + 2];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) return -1;
    o->faces[f][0] = a; o->faces[f][1] = b; o->faces[f][2] = c;
    const double* va = o->bv[a];
    const double* vb = o->bv[b];
    const double* vc = o->bv[c];
    const double e1[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
    const double e2[3] = {vc[0] - va[0], vc[1] - va[1], vc[2] - va[2]};
    const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                          e1[0] * e2[1] - e1[1] * e2[0]};
    const double l = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    if (!(l > 0.0)) return -1;
    o->bn[f][0] = cr[0] / l; o->bn[f][1] = cr[1] / l; o->bn[f][2] = cr[2] / l;
  }
  /* edges: every directed edge (a, b) of a face; (a < b) with both faces */
  int ne = 0;
  for (int f = 0; f < nf; ++f)
    for (int k = 0; k < 3; ++k) {
      const int a = o->faces[f][k], b = o->faces[f][(k + 1) % 3];
      if (a > b) continue;
      int g = -1;
      for (int h = 0; h < nf; ++h)
        for (int q = 0; q < 3; ++q)
          if (o->faces[h][q] == b && o->faces[h][(q + 1) % 3] == a) g = h;
      if (g < 0 || ne >= MIX_E) return -1;
      o->edges[ne][0] = a; o->edges[ne][1] = b;
      o->edges[ne][2] = f < g ? f : g; o->edges[ne][3] = f < g ? g : f;
      ++ne;
    }
  if (ne != 3 * nv - 6) return -1;
  qsort(o->edges, ne, sizeof(o->edges[0]), edge_cmp);
  o->ne = ne;
  double rb = 0.0;
  for (int k = 0; k < nv; ++k) {
    const double r = sqrt(o->bv[k][0] * o->bv[k][0] + o->bv[k][1] * o->bv[k][1] +
                          o->bv[k][2] * o->bv[k][2]);
    if (r > rb) rb = r;
  }
  float rbf = (float)rb;
  if ((double)rbf < rb) rbf = nextafterf(rbf, INFINITY);
  o->rb = rbf;
  double vol = 0.0, cen[3] = {0.0, 0.0, 0.0}, C[9] = {0.0};
  for (int f = 0; f < nf; ++f) {
    const double* a = o->bv[o->faces[f][0]];
    const double* b = o->bv[o->faces[f][1]];
    const double* c = o->bv[o->faces[f][2]];
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
  if (!(vol > 0.0)) return -1;
  const double rho = (double)s->density;
  const double mass = rho * vol;
  double com[3];
  for (int q = 0; q < 3; ++q) com[q] = cen[q] / vol;
  const double tr = C[0] + C[4] + C[8];
  const double c2 = com[0] * com[0] + com[1] * com[1] + com[2] * com[2];
  double J[9];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q)
      J[3 * r + q] = rho * ((r == q ? tr : 0.0) - C[3 * r + q]) -
                     mass * ((r == q ? c2 : 0.0) - com[r] * com[q]);
  const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]);
  if (!(det > 0.0)) return -1;
  const double inv[9] = {(J[4] * J[8] - J[5] * J[7]) / det, (J[2] * J[7] - J[1] * J[8]) / det,
                         (J[1] * J[5] - J[2] * J[4]) / det, (J[5] * J[6] - J[3] * J[8]) / det,
                         (J[0] * J[8] - J[2] * J[6]) / det, (J[2] * J[3] - J[0] * J[5]) / det,
                         (J[3] * J[7] - J[4] * J[6]) / det, (J[1] * J[6] - J[0] * J[7]) / det,
                         (J[0] * J[4] - J[1] * J[3]) / det};
  o->mass = (real)mass;
  for (int q = 0; q < 9; ++q) {
    o->inertia[q] = (real)J[q];
    o->iinv[q] = (real)inv[q];
  }
  return 0;
}

/* After ens_set_state: particle i (caller order) with shape_of[i] >= 0 is a
 * polyhedron of shapes[shape_of[i]] oriented by quat4[4 i ..] (normalised in
 * double, then rounded to float). */
int ens_set_polyhedra(ens_oracle* o, const blaze_shape* shapes, int nshapes, const int* shape_of,
                      const double* quat4) {
  free_mix(o);
  int np = 0;
  for (int i = 0; i < o->n; ++i) np += shape_of[i] >= 0;
  if (np == 0) return 0;
  mixc* m = (mixc*)calloc(1, sizeof(mixc));
  m->nshape = nshapes;
  m->shapes = (mshape*)calloc(nshapes, sizeof(mshape));
  for (int k = 0; k < nshapes; ++k)
    if (mix_shape(&shapes[k], &m->shapes[k])) { free(m->shapes); free(m); return -1; }
  m->npoly = np;
  m->shape_of = (int*)calloc(np, sizeof(int));
  m->quat = (real*)calloc((size_t)4 * np, sizeof(real));
  m->path = (real*)calloc(np, sizeof(real));
  m->pat = (int*)calloc(np, sizeof(int));
  m->gv = (double*)calloc((size_t)np * MIX_V * 4, sizeof(double));
  m->gf = (double*)calloc((size_t)np * MIX_F * 4, sizeof(double));
  m->wh = (real*)calloc((size_t)np * MIX_WSLOTS * 3, sizeof(real));
  m->wid = (int*)calloc((size_t)np * MIX_WSLOTS, sizeof(int));
  m->wn = (int*)calloc(np, sizeof(int));
  for (int c = 0; c < 2; ++c) {
    m->idx[c] = (uint32_t*)calloc((size_t)np * MIX_SLOTS, sizeof(uint32_t));
    m->cnt[c] = (uint32_t*)calloc(np, sizeof(uint32_t));
    m->mask[c] = (uint64_t*)calloc(np, sizeof(uint64_t));
    m->hist[c] = (real*)calloc((size_t)np * MIX_SLOTS * 3, sizeof(real));
  }
  int p = 0;
  for (int i = 0; i < o->n; ++i) {
    if (shape_of[i] < 0) continue;
    const mshape* sh = &m->shapes[shape_of[i]];
    m->shape_of[p] = shape_of[i];
    const double* q = quat4 + 4 * i;
    const double qn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    /* as the product takes it, in both builds: normalised in double, rounded
       to float (a 1-ulp turn moves a vertex by ~1e-7 cm, a few 1e-3 of a
       resting overlap) */
    for (int c = 0; c < 4; ++c) m->quat[4 * p + c] = (real)(float)(q[c] / qn);
    m->pat[p] = i;
    o->p[i].poly = p;
    o->p[i].r = (real)sh->rb;
    ++p;
  }
  o->mix = m;
  return 0;
}

/* Orientations in the current memory order (w x y z; spheres 1 0 0 0). */
void ens_get_orientations(const ens_oracle* o, double* quat4) {
  for (int i = 0; i < o->n; ++i) {
    const int p = o->p[i].poly;
    for (int c = 0; c < 4; ++c)
      quat4[4 * i + c] = p >= 0 ? (double)o->mix->quat[4 * p + c] : (c == 0 ? 1.0 : 0.0);
  }
}

/* FP64 vectors, evaluated as csrc/mix_device.cuh writes them */
typedef struct { double x, y, z; } dv3;
static dv3 dv(double x, double y, double z) { dv3 r = {x, y, z}; return r; }
static dv3 dof(v3 a) { return dv((double)a.x, (double)a.y, (double)a.z); }
static dv3 d4v(const double* p) { return dv(p[0], p[1], p[2]); }
static dv3 dadd(dv3 a, dv3 b) { return dv(a.x + b.x, a.y + b.y, a.z + b.z); }
static dv3 dsub(dv3 a, dv3 b) { return dv(a.x - b.x, a.y - b.y, a.z - b.z); }
static dv3 dscale(dv3 a, double s) { return dv(a.x * s, a.y * s, a.z * s); }
static dv3 dneg(dv3 a) { return dv(-a.x, -a.y, -a.z); }
static double ddot(dv3 a, dv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static dv3 dcross(dv3 a, dv3 b) {
  return dv(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3 tov(dv3 a) { return mk((real)a.x, (real)a.y, (real)a.z); }

static void mix_rotation(const real* q4, double* R) {
  const double w = q4[0], x = q4[1], y = q4[2], z = q4[3];
  const double s = 2.0 / (((w * w + x * x) + y * y) + z * z);
  R[0] = 1.0 - s * (y * y + z * z);
  R[1] = s * (x * y - w * z);
  R[2] = s * (x * z + w * y);
  R[3] = s * (x * y + w * z);
  R[4] = 1.0 - s * (x * x + z * z);
  R[5] = s * (y * z - w * x);
  R[6] = s * (x * z - w * y);
  R[7] = s * (y * z + w * x);
  R[8] = 1.0 - s * (x * x + y * y);
}
static dv3 mat_vec(const double* R, dv3 v) {
  return dv((R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
            (R[6] * v.x + R[7] * v.y) + R[8] * v.z);
}
static dv3 rot_about_d(dv3 a, double c, double s, dv3 v) {
  const dv3 axv = dcross(a, v);
  const double av = ddot(a, v);
  return dadd(dadd(dscale(v, c), dscale(axv, s)), dscale(a, av * (1.0 - c)));
}

static dv3 closest_on_triangle_d(dv3 p, dv3 a, dv3 b, dv3 c) {
  const dv3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
  const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const dv3 bp = dsub(p, b);
  const double d3_ = ddot(ab, bp), d4 = ddot(ac, bp);
  if (d3_ >= 0.0 && d4 <= d3_) return b;
  const double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) return dadd(a, dscale(ab, d1 / (d1 - d3_)));
  const dv3 cp = dsub(p, c);
  const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return dadd(a, dscale(ac, d2 / (d2 - d6)));
  const double va = d3_ * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0)
    return dadd(b, dscale(dsub(c, b), (d4 - d3_) / ((d4 - d3_) + (d5 - d6))));
  const double den = 1.0 / ((va + vb) + vc);
  return dadd(dadd(a, dscale(ab, vb * den)), dscale(ac, vc * den));
}

typedef struct { v3 n; real delta; v3 ca, cb; } mhit;

/* a world-frame hull: vertex offsets V[k * 4], planes F[f * 4] (normal, h) */
typedef struct {
  const double* V;
  const double* F;
  const int (*E)[4];
  const int (*T)[3];
  int nv, nf, ne;
} hullr;

static int sphere_hull(v3 c, real r, v3 x, const hullr* H, mhit* h) {
  const dv3 d = dsub(dof(c), dof(x));
  const double rr = (double)r;
  double smax = -1e300;
  int fb = 0;
  for (int f = 0; f < H->nf; ++f) {
    const double* P = H->F + 4 * f;
    const double s = ((P[0] * d.x + P[1] * d.y) + P[2] * d.z) - P[3];
    if (s > smax) { smax = s; fb = f; }
  }
  if (!(smax < rr)) return 0;
  dv3 q, nn;
  double delta;
  if (smax <= 0.0) {
    nn = d4v(H->F + 4 * fb);
    delta = rr - smax;
    q = dsub(d, dscale(nn, smax));
  } else {
    double best = 1e300;
    q = d;
    for (int f = 0; f < H->nf; ++f) {
      const double* P = H->F + 4 * f;
      const double s = ((P[0] * d.x + P[1] * d.y) + P[2] * d.z) - P[3];
      if (!(s > 0.0 && s < rr)) continue;
      const int* t = H->T[f];
      const dv3 qf = closest_on_triangle_d(d, d4v(H->V + 4 * t[0]), d4v(H->V + 4 * t[1]),
                                           d4v(H->V + 4 * t[2]));
      const dv3 e = dsub(d, qf);
      const double e2 = ddot(e, e);
      if (e2 < best) { best = e2; q = qf; }
    }
    if (!(best < rr * rr)) return 0;
    const double dist = sqrt(best);
    if (!(dist > 0.0)) return 0;
    nn = dv((d.x - q.x) / dist, (d.y - q.y) / dist, (d.z - q.z) / dist);
    delta = rr - dist;
  }
  const real df = (real)delta;
  if (!(df > 0)) return 0;
  h->n = tov(nn);
  h->delta = df;
  h->ca = mul(h->n, -r);
  h->cb = tov(q);
  return 1;
}

static double face_sep(const double* P, dv3 d, const double* VB, int nvB) {
  double m = 1e300;
  for (int k = 0; k < nvB; ++k) {
    const double* v = VB + 4 * k;
    const double t = (P[0] * (d.x + v[0]) + P[1] * (d.y + v[1])) + P[2] * (d.z + v[2]);
    if (t < m) m = t;
  }
  return m - P[3];
}

#define NO_AXIS (-1e300)

static double edge_sep(dv3 a, dv3 b, dv3 c, dv3 dn, dv3 PA, dv3 QA, dv3 PB, dv3 QB) {
  c = dneg(c);
  dn = dneg(dn);
  const dv3 bxa = dcross(b, a), dxc = dcross(dn, c);
  const double cba = ddot(c, bxa), dba = ddot(dn, bxa), adc = ddot(a, dxc), bdc = ddot(b, dxc);
  if (!(cba * dba < 0.0 && adc * bdc < 0.0 && cba * bdc > 0.0)) return NO_AXIS;
  const dv3 ea = dsub(QA, PA), eb = dsub(QB, PB);
  dv3 ax = dcross(ea, eb);
  const double l2 = ddot(ax, ax);
  if (!(l2 > 1e-10 * (ddot(ea, ea) * ddot(eb, eb)))) return NO_AXIS;
  const double l = sqrt(l2);
  ax = dv(ax.x / l, ax.y / l, ax.z / l);
  if (ddot(ax, PA) < 0.0) ax = dneg(ax);
  return ddot(ax, dsub(PB, PA));
}

static dv3 edge_axis(dv3 PA, dv3 QA, dv3 PB, dv3 QB) {
  const dv3 ea = dsub(QA, PA), eb = dsub(QB, PB);
  dv3 ax = dcross(ea, eb);
  const double l = sqrt(ddot(ax, ax));
  ax = dv(ax.x / l, ax.y / l, ax.z / l);
  if (ddot(ax, PA) < 0.0) ax = dneg(ax);
  return ax;
}

static double clamp01(double s) { return s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s); }

static dv3 segments_midpoint(dv3 P1, dv3 Q1, dv3 P2, dv3 Q2) {
  const dv3 d1 = dsub(Q1, P1), d2 = dsub(Q2, P2), r = dsub(P1, P2);
  const double a = ddot(d1, d1), e = ddot(d2, d2), f = ddot(d2, r);
  const double c = ddot(d1, r), b = ddot(d1, d2);
  const double den = a * e - b * b;
  double s = den > 0.0 ? (b * f - c * e) / den : 0.0;
  s = clamp01(s);
  double t = (b * s + f) / e;
  if (t < 0.0) {
    t = 0.0;
    s = clamp01(-c / a);
  } else if (t > 1.0) {
    t = 1.0;
    s = clamp01((b - c) / a);
  }
  const dv3 c1 = dadd(P1, dscale(d1, s)), c2 = dadd(P2, dscale(d2, t));
  return dscale(dadd(c1, c2), 0.5);
}

#define REL_FACE 0.98
#define REL_EDGE 0.90

typedef struct { double sA, sB, sE; int fA, fB, eE; } satpick;

static int sat_kind(const satpick* q) {
  const double sf = q->sA > q->sB ? q->sA : q->sB;
  if (q->sE > REL_EDGE * sf) return 2;
  if (q->sB > REL_FACE * q->sA) return 1;
  return 0;
}

/* the separating-axis queries of A and B (B's centre at d from A's) */
static int hull_hull_queries(dv3 d, const hullr* A, const hullr* B, satpick* q) {
  double s = -1e300;
  int k = 0;
  for (int f = 0; f < A->nf; ++f) {
    const double t = face_sep(A->F + 4 * f, d, B->V, B->nv);
    if (t > s) { s = t; k = f; }
  }
  if (s > 0.0) return 0;
  q->sA = s; q->fA = k;
  const dv3 md = dneg(d);
  s = -1e300;
  k = 0;
  for (int f = 0; f < B->nf; ++f) {
    const double t = face_sep(B->F + 4 * f, md, A->V, A->nv);
    if (t > s) { s = t; k = f; }
  }
  if (s > 0.0) return 0;
  q->sB = s; q->fB = k;
  s = NO_AXIS;
  k = 0;
  for (int ea = 0; ea < A->ne; ++ea)
    for (int eb = 0; eb < B->ne; ++eb) {
      const int* EA = A->E[ea];
      const int* EB = B->E[eb];
      const double t = edge_sep(d4v(A->F + 4 * EA[2]), d4v(A->F + 4 * EA[3]), d4v(B->F + 4 * EB[2]),
                                d4v(B->F + 4 * EB[3]), d4v(A->V + 4 * EA[0]), d4v(A->V + 4 * EA[1]),
                                dadd(d, d4v(B->V + 4 * EB[0])), dadd(d, d4v(B->V + 4 * EB[1])));
      if (t > s) { s = t; k = ea * B->ne + eb; }
    }
  if (s > 0.0) return 0;
  q->sE = s; q->eE = k;
  return 1;
}

static int hull_hull_finish(const satpick* q, dv3 d, const hullr* A, const hullr* B, mhit* h) {
  const int kind = sat_kind(q);
  dv3 nAB, cp;
  double s;
  if (kind == 0) {
    const double* P = A->F + 4 * q->fA;
    nAB = d4v(P);
    s = q->sA;
    dv3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < B->nv; ++k) {
      const dv3 v = dadd(d, d4v(B->V + 4 * k));
      const double t = ((P[0] * v.x + P[1] * v.y) + P[2] * v.z) - P[3];
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else if (kind == 1) {
    const double* P = B->F + 4 * q->fB;
    nAB = dneg(d4v(P));
    s = q->sB;
    dv3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < A->nv; ++k) {
      const dv3 v = d4v(A->V + 4 * k);
      const dv3 w = dsub(v, d);
      const double t = ((P[0] * w.x + P[1] * w.y) + P[2] * w.z) - P[3];
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else {
    const int* ea = A->E[q->eE / B->ne];
    const int* eb = B->E[q->eE % B->ne];
    const dv3 PA = d4v(A->V + 4 * ea[0]), QA = d4v(A->V + 4 * ea[1]);
    const dv3 PB = dadd(d, d4v(B->V + 4 * eb[0])), QB = dadd(d, d4v(B->V + 4 * eb[1]));
    nAB = edge_axis(PA, QA, PB, QB);
    s = q->sE;
    cp = segments_midpoint(PA, QA, PB, QB);
  }
  const real df = (real)(-s);
  if (!(df > 0)) return 0;
  h->n = tov(dneg(nAB));
  h->delta = df;
  h->ca = tov(cp);
  h->cb = tov(dsub(cp, d));
  return 1;
}

static int tri_e0(int t) { return t == 2 ? 1 : 0; }
static int tri_e1(int t) { return t == 0 ? 1 : 2; }

static int hull_tri(const hullr* H, const dv3* T, dv3 nt, mhit* h, dv3* nd, int* kind_out) {
  double sP = -1e300;
  int fP = 0;
  for (int f = 0; f < H->nf; ++f) {
    const double* P = H->F + 4 * f;
    double m = 1e300;
    for (int k = 0; k < 3; ++k) {
      const double t = (P[0] * T[k].x + P[1] * T[k].y) + P[2] * T[k].z;
      if (t < m) m = t;
    }
    const double s = m - P[3];
    if (s > sP) { sP = s; fP = f; }
  }
  if (sP > 0.0) return 0;
  double lo = 1e300, hi = -1e300;
  for (int k = 0; k < H->nv; ++k) {
    const double t = ddot(nt, d4v(H->V + 4 * k));
    if (t < lo) lo = t;
    if (t > hi) hi = t;
  }
  const double h0 = ddot(nt, T[0]);
  const double sTp = lo - h0, sTm = h0 - hi;
  const int tplus = sTp >= sTm;
  const double sT = tplus ? sTp : sTm;
  if (sT > 0.0) return 0;
  double sE = -1e300;
  int eE = -1, eplus = 1;
  for (int e = 0; e < H->ne; ++e) {
    const int* ed = H->E[e];
    const dv3 P0 = d4v(H->V + 4 * ed[0]), ep = dsub(d4v(H->V + 4 * ed[1]), P0);
    for (int t = 0; t < 3; ++t) {
      const dv3 et = dsub(T[tri_e1(t)], T[tri_e0(t)]);
      dv3 ax = dcross(ep, et);
      const double l2 = ddot(ax, ax);
      if (!(l2 > 1e-10 * (ddot(ep, ep) * ddot(et, et)))) continue;
      const double l = sqrt(l2);
      ax = dv(ax.x / l, ax.y / l, ax.z / l);
      double pmin = 1e300, pmax = -1e300;
      for (int k = 0; k < H->nv; ++k) {
        const double u = ddot(ax, d4v(H->V + 4 * k));
        if (u < pmin) pmin = u;
        if (u > pmax) pmax = u;
      }
      double tmin = 1e300, tmax = -1e300;
      for (int k = 0; k < 3; ++k) {
        const double u = ddot(ax, T[k]);
        if (u < tmin) tmin = u;
        if (u > tmax) tmax = u;
      }
      const double s1 = tmin - pmax, s2 = pmin - tmax;
      const double s = s1 >= s2 ? s1 : s2;
      if (s > 0.0) return 0;
      if (s > sE) { sE = s; eE = 3 * e + t; eplus = s1 >= s2; }
    }
  }
  satpick q;
  q.sA = sT;
  q.sB = sP;
  q.sE = eE >= 0 ? sE : NO_AXIS;
  const int kind = sat_kind(&q);
  dv3 n_in, cp;
  double s;
  if (kind == 0) {
    n_in = tplus ? nt : dneg(nt);
    s = sT;
    dv3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < H->nv; ++k) {
      const dv3 v = d4v(H->V + 4 * k);
      const double t = ddot(n_in, v) - ddot(n_in, T[0]);
      if (t < 0.0) { acc = dadd(acc, dscale(v, -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else if (kind == 1) {
    const double* P = H->F + 4 * fP;
    n_in = dneg(d4v(P));
    s = sP;
    dv3 acc = dv(0.0, 0.0, 0.0);
    double wsum = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double t = ((P[0] * T[k].x + P[1] * T[k].y) + P[2] * T[k].z) - P[3];
      if (t < 0.0) { acc = dadd(acc, dscale(T[k], -t)); wsum = wsum - t; }
    }
    cp = dscale(acc, 1.0 / wsum);
  } else {
    const int e = eE / 3, t = eE % 3;
    const int* ed = H->E[e];
    const dv3 P0 = d4v(H->V + 4 * ed[0]), Q0 = d4v(H->V + 4 * ed[1]);
    const dv3 P1 = T[tri_e0(t)], Q1 = T[tri_e1(t)];
    dv3 ax = dcross(dsub(Q0, P0), dsub(Q1, P1));
    const double l = sqrt(ddot(ax, ax));
    ax = dv(ax.x / l, ax.y / l, ax.z / l);
    n_in = eplus ? dneg(ax) : ax;
    s = sE;
    cp = segments_midpoint(P0, Q0, P1, Q1);
  }
  const real df = (real)(-s);
  if (!(df > 0)) return 0;
  *nd = n_in;
  *kind_out = kind;
  h->n = tov(n_in);
  h->delta = df;
  h->ca = tov(cp);
  h->cb = h->ca;
  return 1;
}

static int hull_plane(v3 n, real pd, v3 x, const hullr* H, mhit* h) {
  const dv3 nn = dof(n);
  const double base = ddot(nn, dof(x)) - (double)pd;
  double lo = 1e300, wsum = 0.0;
  dv3 acc = dv(0.0, 0.0, 0.0);
  for (int k = 0; k < H->nv; ++k) {
    const dv3 v = d4v(H->V + 4 * k);
    const double s = base + ddot(nn, v);
    if (s < lo) lo = s;
    if (s < 0.0) { acc = dadd(acc, dscale(v, -s)); wsum = wsum - s; }
  }
  const real df = (real)(-lo);
  if (!(df > 0) || !(wsum > 0.0)) return 0;
  h->n = n;
  h->delta = df;
  h->ca = tov(dscale(acc, 1.0 / wsum));
  h->cb = h->ca;
  return 1;
}

#define COPLANAR (1.0 - 1e-9)

static hullr hull_of(const mixc* m, int p) {
  const mshape* sh = &m->shapes[m->shape_of[p]];
  hullr h;
  h.V = m->gv + (size_t)p * MIX_V * 4;
  h.F = m->gf + (size_t)p * MIX_F * 4;
  h.E = (const int (*)[4])sh->edges;
  h.T = (const int (*)[3])sh->faces;
  h.nv = sh->nv;
  h.nf = sh->nf;
  h.ne = sh->ne;
  return h;
}

/* world-frame geometry of every polyhedron from its orientation (k_mix_geom) */
static void mix_geometry(ens_oracle* o) {
  mixc* m = o->mix;
  for (int p = 0; p < m->npoly; ++p) {
    const mshape* sh = &m->shapes[m->shape_of[p]];
    double R[9];
    mix_rotation(m->quat + 4 * p, R);
    double* V = m->gv + (size_t)p * MIX_V * 4;
    double* F = m->gf + (size_t)p * MIX_F * 4;
    for (int k = 0; k < sh->nv; ++k) {
      const dv3 v = mat_vec(R, d4v(sh->bv[k]));
      V[4 * k] = v.x; V[4 * k + 1] = v.y; V[4 * k + 2] = v.z; V[4 * k + 3] = 0.0;
    }
    for (int f = 0; f < sh->nf; ++f) {
      const dv3 n = mat_vec(R, d4v(sh->bn[f]));
      const dv3 v = mat_vec(R, d4v(sh->bv[sh->faces[f][0]]));
      F[4 * f] = n.x; F[4 * f + 1] = n.y; F[4 * f + 2] = n.z; F[4 * f + 3] = ddot(n, v);
    }
  }
}

/* The law of a contact h of particle a with particle b (mix_pair_law). */
static void mix_pair_law(const ens_oracle* o, const sysc* S, const mhit* h, real ma, v3 va, v3 wa,
                         real mb, v3 vb, v3 wb, v3* xi, v3* F, v3* Ta, v3* Tb) {
  const v3 vct = sub(add(va, cross(wa, h->ca)), add(vb, cross(wb, h->cb)));
  const real ms = (ma * mb) / (ma + mb);
  v3 t0;
  contact_law(o, S, S->mu, h->n, h->delta, 0, ms, vct, vct, mk(0, 0, 0), 0, xi, F, &t0);
  *Ta = cross(h->ca, *F);
  *Tb = cross(h->cb, mk(-F->x, -F->y, -F->z));
}

/* The polyhedra's lists of the new memory order (k_mix_plist), after the
 * re-sort placed them: the new order is o->q, the old o->p. */
static void mix_rebuild_lists(ens_oracle* o) {
  mixc* m = o->mix;
  const int n = o->n, e = o->epoch & 1;
  const size_t P = (size_t)m->npoly;
  for (int i = 0; i < n; ++i)
    if (o->q[i].poly >= 0) {
      m->pat[o->q[i].poly] = i;
      m->path[o->q[i].poly] = 0;
    }
  uint32_t *Io = m->idx[e], *In = m->idx[e ^ 1];
  uint32_t *Co = m->cnt[e], *Cn = m->cnt[e ^ 1];
  uint64_t *Mo = m->mask[e], *Mn = m->mask[e ^ 1];
  real *Ho = m->hist[e], *Hn = m->hist[e ^ 1];
  for (int p = 0; p < m->npoly; ++p) {
    const int i = m->pat[p];
    const part* a = &o->q[i];
    const sysc* S = &o->S[a->sys];
    const uint32_t cnt_o = Co[p];
    const uint64_t mask_o = Mo[p];
    uint32_t cnt = 0;
    uint64_t mask = 0;
    int c[3];
    if (cell_of(S, a->pos, c)) {
      const int x0 = c[0] > 0 ? c[0] - 1 : 0, x1 = c[0] < S->nc[0] - 1 ? c[0] + 1 : c[0];
      const int y0 = c[1] > 0 ? c[1] - 1 : 0, y1 = c[1] < S->nc[1] - 1 ? c[1] + 1 : c[1];
      const int z0 = c[2] > 0 ? c[2] - 1 : 0, z1 = c[2] < S->nc[2] - 1 ? c[2] + 1 : c[2];
      for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
          for (int x = x0; x <= x1; ++x) {
            const uint32_t h = S->cell_off + (uint32_t)(S->nc[0] * (y + S->nc[1] * z)) + (uint32_t)x;
            const uint32_t s0 = o->cstart[h];
            if (s0 == 0xffffffffu) continue;
            for (uint32_t j = s0; j < o->cend[h]; ++j) {
              if ((int)j == i) continue;
              const part* b = &o->q[j];
              const v3 rel = sub(a->pos, b->pos);
              const real lim = (a->r + b->r) + o->skin;
              if (!(dot(rel, rel) < lim * lim)) continue;
              if (cnt < MIX_SLOTS) {
                In[(size_t)cnt * P + p] = j;
                for (uint32_t ko = 0; ko < cnt_o && ko < MIX_SLOTS; ++ko) {
                  if (!((mask_o >> ko) & 1ull)) continue;
                  const size_t so = (size_t)ko * P + p;
                  if (o->p[Io[so]].pid == b->pid) {
                    const size_t sn = (size_t)cnt * P + p;
                    Hn[3 * sn] = Ho[3 * so]; Hn[3 * sn + 1] = Ho[3 * so + 1]; Hn[3 * sn + 2] = Ho[3 * so + 2];
                    mask |= 1ull << cnt;
                    break;
                  }
                }
              } else {
                o->status |= ST_OVERFLOW;
              }
              ++cnt;
            }
          }
    } else {
      o->status |= ST_OUT_OF_GRID;
    }
    Cn[p] = cnt < MIX_SLOTS ? cnt : MIX_SLOTS;
    Mn[p] = mask;
  }
}

/* One sphere's contact with polyhedron neighbour b (the sphere step's
 * branch); 0 when they do not touch. */
static int mix_sphere_contact(const ens_oracle* o, const sysc* S, const part* a, real ma,
                              const part* b, v3* xi, v3* F, v3* T) {
  const mixc* m = o->mix;
  const hullr H = hull_of(m, b->poly);
  mhit h;
  if (!sphere_hull(a->pos, a->r, b->pos, &H, &h)) return 0;
  v3 Tb;
  mix_pair_law(o, S, &h, ma, a->vel, a->w, m->shapes[m->shape_of[b->poly]].mass, b->vel, b->w, xi,
               F, T, &Tb);
  return 1;
}

enum { MIX_HITS = 32 };

/* One polyhedron's step (k_mix_poly_step): reads o->p, writes o->q. */
static void mix_poly_step(ens_oracle* o, int p, int* req) {
  mixc* m = o->mix;
  const int e = o->epoch & 1;
  const size_t P = (size_t)m->npoly;
  const int i = m->pat[p];
  const part* a = &o->p[i];
  const sysc* S = &o->S[a->sys];
  const mshape* SH = &m->shapes[m->shape_of[p]];
  const hullr A = hull_of(m, p);
  const real dt = o->dt;
  uint32_t* I = m->idx[e];
  real* Hs = m->hist[e];
  const uint32_t cnt = m->cnt[e][p];
  const uint64_t mask_o = m->mask[e][p];
  uint64_t touch = 0;
  v3 f = mk(0, 0, 0), t = mk(0, 0, 0);
  for (uint32_t k = 0; k < cnt; ++k) {
    const size_t sk = (size_t)k * P + p;
    const part* b = &o->p[I[sk]];
    v3 xi = mk(0, 0, 0);
    if ((mask_o >> k) & 1ull) xi = mk(Hs[3 * sk], Hs[3 * sk + 1], Hs[3 * sk + 2]);
    v3 F, Ta, Tb;
    if (b->poly < 0) {
      const v3 rel = sub(b->pos, a->pos);
      const real sr = b->r + a->r;
      const real d2 = dot(rel, rel);
      if (!(d2 < sr * sr && SQRT(d2) > 0)) continue;
      mhit h;
      if (!sphere_hull(b->pos, b->r, a->pos, &A, &h)) continue;
      const real mb = S->dens43pi * ((b->r * b->r) * b->r);
      mix_pair_law(o, S, &h, mb, b->vel, b->w, SH->mass, a->vel, a->w, &xi, &F, &Ta, &Tb);
      f = add(f, mk(-F.x, -F.y, -F.z));
      t = add(t, Tb);
    } else {
      const int q = b->poly;
      const int selfA = p < q;
      const part* pA = selfA ? a : b;
      const part* pB = selfA ? b : a;
      const v3 rel = sub(pB->pos, pA->pos);
      const real sr = pA->r + pB->r;
      if (!(dot(rel, rel) < sr * sr)) continue;
      const hullr Bq = hull_of(m, q);
      const hullr* HA = selfA ? &A : &Bq;
      const hullr* HB = selfA ? &Bq : &A;
      const dv3 d = dsub(dof(pB->pos), dof(pA->pos));
      satpick pk;
      if (!hull_hull_queries(d, HA, HB, &pk)) continue;
      mhit h;
      if (!hull_hull_finish(&pk, d, HA, HB, &h)) continue;
      const real mq = m->shapes[m->shape_of[q]].mass;
      if (selfA) mix_pair_law(o, S, &h, SH->mass, a->vel, a->w, mq, b->vel, b->w, &xi, &F, &Ta, &Tb);
      else mix_pair_law(o, S, &h, mq, b->vel, b->w, SH->mass, a->vel, a->w, &xi, &F, &Ta, &Tb);
      f = add(f, selfA ? F : mk(-F.x, -F.y, -F.z));
      t = add(t, selfA ? Ta : Tb);
    }
    Hs[3 * sk] = xi.x; Hs[3 * sk + 1] = xi.y; Hs[3 * sk + 2] = xi.z;
    touch |= 1ull << k;
  }
  m->mask[e][p] = touch;

  /* walls */
  part* out = &o->q[i];
  *out = *a;
  int nw = 0;
  uint32_t st = 0;
  const int rot = S->rot;
  const real rc = o->rot_c[a->sys], rsn = o->rot_s[a->sys];
  /* the polyhedron's wall histories (by wall id), new ones in processing order */
  real* wh = m->wh + (size_t)p * MIX_WSLOTS * 3;
  int* wid = m->wid + (size_t)p * MIX_WSLOTS;
  const int nw_o = m->wn[p];
  real oh[MIX_WSLOTS][3];
  int oid[MIX_WSLOTS];
  for (int q_ = 0; q_ < MIX_WSLOTS; ++q_) {
    oid[q_] = q_ < nw_o ? wid[q_] : -1;
    for (int c_ = 0; c_ < 3; ++c_) oh[q_][c_] = q_ < nw_o ? wh[3 * q_ + c_] : 0;
  }
#define MIX_WALL(ID, H, MOVING)                                                               \
  do {                                                                                        \
    v3 xi_ = mk(0, 0, 0);                                                                     \
    for (int q_ = 0; q_ < MIX_WSLOTS; ++q_)                                                   \
      if (oid[q_] == (ID)) xi_ = mk(oh[q_][0], oh[q_][1], oh[q_][2]);                         \
    const v3 vw_ = (MOVING) ? mul(cross(S->rot_a, sub(add(a->pos, (H).ca), S->rot_o)), S->rot_w) \
                            : mk(0, 0, 0);                                                    \
    const v3 vct_ = sub(add(a->vel, cross(a->w, (H).ca)), vw_);                               \
    v3 F_, t0_;                                                                               \
    contact_law(o, S, S->mu_w, (H).n, (H).delta, 0, SH->mass, vct_, vct_, mk(0, 0, 0), 0, &xi_, \
                &F_, &t0_);                                                                   \
    f = add(f, F_);                                                                           \
    t = add(t, cross((H).ca, F_));                                                            \
    if (nw < MIX_WSLOTS) {                                                                    \
      wh[3 * nw] = xi_.x; wh[3 * nw + 1] = xi_.y; wh[3 * nw + 2] = xi_.z;                     \
      wid[nw] = (ID);                                                                         \
      ++nw;                                                                                   \
    } else {                                                                                  \
      st |= ST_OVERFLOW;                                                                      \
    }                                                                                         \
  } while (0)
  for (int w = S->wall0; w < S->wall0 + S->nwall; ++w) {
    const wallc* W = &o->W[w];
    mhit h;
    if (W->kind == BLAZE_WALL_PLANE && hull_plane(W->a, W->r, a->pos, &A, &h))
      MIX_WALL(w, h, rot && W->turning);
  }
  int cc[3];
  const v3 pd = rot ? add(S->rot_o, rot_about(S->rot_a, rc, -rsn, sub(a->pos, S->rot_o))) : a->pos;
  if (S->ntri > 0 && cell_of(S, pd, cc)) {
    const uint32_t tq0 = o->use_tri_lists ? o->tri_off[key_of(S, cc)] : 0u;
    const uint32_t tq1 = o->use_tri_lists ? o->tri_off[key_of(S, cc) + 1] : (uint32_t)S->ntri;
    /* the polyhedron in the drum's frame */
    double Vd[MIX_V * 4], Fd[MIX_F * 4];
    hullr D = A;
    if (rot) {
      const dv3 ax = dof(S->rot_a);
      const double c = (double)rc, s = -(double)rsn;
      for (int k = 0; k < A.nv; ++k) {
        const dv3 v = rot_about_d(ax, c, s, d4v(A.V + 4 * k));
        Vd[4 * k] = v.x; Vd[4 * k + 1] = v.y; Vd[4 * k + 2] = v.z; Vd[4 * k + 3] = 0.0;
      }
      for (int f2 = 0; f2 < A.nf; ++f2) {
        const dv3 nn = rot_about_d(ax, c, s, d4v(A.F + 4 * f2));
        Fd[4 * f2] = nn.x; Fd[4 * f2 + 1] = nn.y; Fd[4 * f2 + 2] = nn.z; Fd[4 * f2 + 3] = A.F[4 * f2 + 3];
      }
      D.V = Vd;
      D.F = Fd;
    }
    const real lim = (real)SH->rb * (real)1.001f + (real)1e-3f;
    mhit hits[MIX_HITS];
    dv3 nds[MIX_HITS];
    int ids[MIX_HITS], kinds[MIX_HITS], nhit = 0;
    for (uint32_t q_ = tq0; q_ < tq1; ++q_) {
      const int w = o->use_tri_lists ? (int)o->tri_ids[q_] : S->tri0 + (int)q_;
      const wallc* W = &o->W[w];
      int reg, feat;
      const v3 cp = closest_tri(pd, W->a, W->b, W->c, &reg, &feat);
      const v3 dd = sub(pd, cp);
      if (!(dot(dd, dd) < lim * lim)) continue;
      const dv3 o0 = dof(pd);
      dv3 T[3];
      T[0] = dsub(dof(W->a), o0);
      T[1] = dsub(dof(W->b), o0);
      T[2] = dsub(dof(W->c), o0);
      mhit h;
      dv3 nd;
      int kind;
      if (!hull_tri(&D, T, d4v(W->n64), &h, &nd, &kind)) continue;
      if (nhit < MIX_HITS) {
        hits[nhit] = h;
        nds[nhit] = nd;
        ids[nhit] = w;
        kinds[nhit] = kind;
        ++nhit;
      } else {
        st |= ST_OVERFLOW;
      }
    }
    /* face contacts all count, one per plane (the deepest); without one,
       only the deepest other contact does */
    int anyface = 0, best = -1;
    for (int q = 0; q < nhit; ++q) {
      if (kinds[q] == 0) anyface = 1;
      else if (best < 0 || hits[q].delta > hits[best].delta) best = q;
    }
    for (int q = 0; q < nhit; ++q) {
      int keep = anyface ? kinds[q] == 0 : q == best;
      for (int c2 = 0; c2 < nhit && keep && anyface; ++c2) {
        if (c2 == q || kinds[c2] != 0 || !(ddot(nds[q], nds[c2]) > COPLANAR)) continue;
        const real da = hits[q].delta, dc = hits[c2].delta;
        if (dc > da || (dc == da && ids[c2] < ids[q])) keep = 0;
      }
      if (!keep) continue;
      mhit h = hits[q];
      if (rot) {
        h.n = rot_about(S->rot_a, rc, rsn, h.n);
        h.ca = rot_about(S->rot_a, rc, rsn, h.ca);
      }
      MIX_WALL(ids[q], h, rot);
    }
  }
#undef MIX_WALL
  o->status |= st;
  m->wn[p] = nw;
  out->wmask = 0;

  /* translation; Euler's equations in the body frame; the quaternion */
  const real inv_m = (real)1.0 / SH->mass;
  const v3 acc = add(mul(f, inv_m), S->g);
  const v3 v = add(a->vel, mul(acc, dt));
  const v3 x = add(a->pos, mul(v, dt));
  real* qq = m->quat + 4 * p;
  const real qw = qq[0], qx = qq[1], qy = qq[2], qz = qq[3];
  real R[9];
  {
    const real s = (real)2.0 / (((qw * qw + qx * qx) + qy * qy) + qz * qz);
    R[0] = (real)1.0 - s * (qy * qy + qz * qz);
    R[1] = s * (qx * qy - qw * qz);
    R[2] = s * (qx * qz + qw * qy);
    R[3] = s * (qx * qy + qw * qz);
    R[4] = (real)1.0 - s * (qx * qx + qz * qz);
    R[5] = s * (qy * qz - qw * qx);
    R[6] = s * (qx * qz - qw * qy);
    R[7] = s * (qy * qz + qw * qx);
    R[8] = (real)1.0 - s * (qx * qx + qy * qy);
  }
#define MV(M, u) mk(((M)[0] * (u).x + (M)[1] * (u).y) + (M)[2] * (u).z, \
                    ((M)[3] * (u).x + (M)[4] * (u).y) + (M)[5] * (u).z, \
                    ((M)[6] * (u).x + (M)[7] * (u).y) + (M)[8] * (u).z)
#define MTV(M, u) mk(((M)[0] * (u).x + (M)[3] * (u).y) + (M)[6] * (u).z, \
                     ((M)[1] * (u).x + (M)[4] * (u).y) + (M)[7] * (u).z, \
                     ((M)[2] * (u).x + (M)[5] * (u).y) + (M)[8] * (u).z)
  const v3 tb = MTV(R, t), wb = MTV(R, a->w);
  const v3 lb = MV(SH->inertia, wb);
  const v3 rhs = sub(tb, cross(wb, lb));
  const v3 dwb = MV(SH->iinv, rhs);
  const v3 wb2 = add(wb, mul(dwb, dt));
  const v3 w = MV(R, wb2);
#undef MV
#undef MTV
  const real hdt = (real)0.5 * dt;
  const real nw_ = -((w.x * qx + w.y * qy) + w.z * qz);
  const v3 nv_ = add(mk(qw * w.x, qw * w.y, qw * w.z), cross(w, mk(qx, qy, qz)));
  real q2w = qw + hdt * nw_, q2x = qx + hdt * nv_.x, q2y = qy + hdt * nv_.y, q2z = qz + hdt * nv_.z;
  const real qi = (real)1.0 / SQRT(((q2w * q2w + q2x * q2x) + q2y * q2y) + q2z * q2z);
  qq[0] = q2w * qi; qq[1] = q2x * qi; qq[2] = q2y * qi; qq[3] = q2z * qi;
  const real path = m->path[p] + len(v) * dt;
  m->path[p] = path;
  out->pos = x;
  out->vel = v;
  out->w = w;
  if (!(isfinite((double)x.x) && isfinite((double)x.y) && isfinite((double)x.z)))
    o->status |= ST_NONFINITE;
  if (path > (real)0.5 * o->skin) *req = 1;
  o->cap_f[i] = f;
  o->cap_t[i] = t;
}

/* One recorded step of the reverse sweep's tape: the step's input state
 * (after its re-sort), the list it used with masks and histories before the
 * step, and for a re-sort step the permutation and history sources. */
typedef struct tstep_ {
  int rebuilt;
  int* perm;
  int* src;
  part* p;
  uint32_t* idx;
  uint32_t* cnt;
  uint32_t* mask;
  real* hist;
} tstep;

static void step_once_rec(ens_oracle* o, tstep* t);
static void step_once(ens_oracle* o) { step_once_rec(o, NULL); }
static void step_once_rec(ens_oracle* o, tstep* t) {
  const int n = o->n;
  const int rebuilt = o->rebuild_req;
  o->rebuild_req = 0;
  if (rebuilt) rebuild_rec(o, t ? t->perm : NULL, t ? t->src : NULL);
  const int e = o->epoch & 1;
  uint32_t* I = o->idx[e];
  uint32_t* C = o->cnt[e];
  uint32_t* M = o->mask[e];
  real* H = o->hist[e];
  if (t) {
    t->rebuilt = rebuilt;
    memcpy(t->p, o->p, sizeof(part) * n);
    memcpy(t->idx, I, sizeof(uint32_t) * (size_t)o->cap * n);
    memcpy(t->cnt, C, sizeof(uint32_t) * n);
    memcpy(t->mask, M, sizeof(uint32_t) * n);
    memcpy(t->hist, H, sizeof(real) * 3 * (size_t)o->cap * n);
  }
  const real dt = o->dt;
  int req = 0;
  if (o->mix) mix_geometry(o);
  for (int i = 0; i < n; ++i) {
    const part* a = &o->p[i];
    if (a->poly >= 0) continue;   /* stepped by mix_poly_step */
    const sysc* S = &o->S[a->sys];
    const real ra = a->r;
    const real ma = S->dens43pi * ((ra * ra) * ra);
    v3 f = mk(0, 0, 0), t = mk(0, 0, 0);
    uint32_t mask = 0;
    for (uint32_t k = 0; k < C[i]; ++k) {
      const size_t sk = (size_t)k * n + i;
      const part* b = &o->p[I[sk]];
      const v3 rel = sub(a->pos, b->pos);
      const real rb = b->r;
      const real sr = ra + rb;
      const real d2 = dot(rel, rel);
      if (!(d2 < sr * sr)) continue;
      const real dist = SQRT(d2);
      if (!(dist > 0)) continue;
      if (b->poly >= 0) {
        v3 xi = mk(0, 0, 0);
        if ((M[i] >> k) & 1u) xi = mk(H[3 * sk], H[3 * sk + 1], H[3 * sk + 2]);
        v3 F, T;
        if (!mix_sphere_contact(o, S, a, ma, b, &xi, &F, &T)) continue;
        H[3 * sk] = xi.x; H[3 * sk + 1] = xi.y; H[3 * sk + 2] = xi.z;
        mask |= 1u << k;
        f = add(f, F);
        t = add(t, T);
        continue;
      }
      const v3 nrm = mul(rel, (real)1.0 / dist);
      const real delta = overlap_pair(ra, rb, a->pos, b->pos);
      if (!(delta > 0)) continue;
      const real mb = S->dens43pi * ((rb * rb) * rb);
      v3 xi = mk(0, 0, 0);
      if ((M[i] >> k) & 1u) xi = mk(H[3 * sk], H[3 * sk + 1], H[3 * sk + 2]);
      const real rs = (ra * rb) / (ra + rb);
      const real ms = (ma * mb) / (ma + mb);
      const v3 vcpa = add(a->vel, cross(a->w, mul(nrm, -ra)));
      const v3 vcpb = add(b->vel, cross(b->w, mul(nrm, rb)));
      v3 F, T;
      contact_law(o, S, S->mu, nrm, delta, rs, ms, sub(a->vel, b->vel), sub(vcpa, vcpb),
                  sub(a->w, b->w), ra, &xi, &F, &T);
      H[3 * sk] = xi.x; H[3 * sk + 1] = xi.y; H[3 * sk + 2] = xi.z;
      mask |= 1u << k;
      f = add(f, F);
      t = add(t, T);
    }
    M[i] = mask;
    wctx c;
    memset(&c, 0, sizeof(c));
    c.o = o; c.S = S; c.a = a; c.ma = ma; c.f = f; c.t = t;
    for (int w = S->wall0; w < S->wall0 + S->nwall; ++w) {
      v3 nn; real d; int reg;
      if (wall_touch(&o->W[w], a->pos, ra, &nn, &d, &reg))
        wall_contact(&c, w, nn, d, S->rot && o->W[w].turning);
    }
    int cc[3];
    /* a turning drum: its triangles are tested in the drum's frame */
    const real rc = o->rot_c[a->sys], rsn = o->rot_s[a->sys];
    const v3 pd = S->rot ? add(S->rot_o, rot_about(S->rot_a, rc, -rsn, sub(a->pos, S->rot_o)))
                         : a->pos;
    if (S->ntri > 0 && cell_of(S, pd, cc)) {
    const uint32_t tq0 = o->use_tri_lists ? o->tri_off[key_of(S, cc)] : 0u;
    const uint32_t tq1 = o->use_tri_lists ? o->tri_off[key_of(S, cc) + 1] : (uint32_t)S->ntri;
      int nface = 0, best = -1;
      real best_d = 0;
      for (uint32_t q_ = tq0; q_ < tq1; ++q_) {
      const int w = o->use_tri_lists ? (int)o->tri_ids[q_] : S->tri0 + (int)q_;
        v3 nn; real d; int reg;
        if (!wall_touch(&o->W[w], pd, ra, &nn, &d, &reg)) continue;
        if (reg == 0) ++nface;
        else if (best < 0 || d > best_d) { best = w; best_d = d; }
      }
      for (uint32_t q_ = tq0; q_ < tq1; ++q_) {
      const int w = o->use_tri_lists ? (int)o->tri_ids[q_] : S->tri0 + (int)q_;
        v3 nn; real d; int reg;
        if (!wall_touch(&o->W[w], pd, ra, &nn, &d, &reg)) continue;
        if ((nface > 0 && reg == 0) || (nface == 0 && w == best))
          wall_contact(&c, w, S->rot ? rot_about(S->rot_a, rc, rsn, nn) : nn, d, S->rot);
      }
    }
    f = c.f; t = c.t;
    o->status |= c.st;
    part* out = &o->q[i];
    *out = *a;
    for (int q = 0; q < c.nw; ++q) {
      out->wh[q][0] = c.nh[q][0]; out->wh[q][1] = c.nh[q][1]; out->wh[q][2] = c.nh[q][2];
      out->wid[q] = c.nid[q];
    }
    out->wmask = c.nw >= WSLOTS ? (1u << WSLOTS) - 1u : (1u << c.nw) - 1u;
    const real inv_m = (real)1.0 / ma;
    const v3 acc = add(mul(f, inv_m), S->g);
    const v3 v = add(a->vel, mul(acc, dt));
    const v3 p = add(a->pos, mul(v, dt));
    const real inertia = ((real)0.4 * ma) * (ra * ra);
    const v3 w = add(a->w, mul(mul(t, (real)1.0 / inertia), dt));
    out->pos = p;
    out->vel = v;
    out->w = w;
    out->path = a->path + len(v) * dt;
    if (!(isfinite((double)p.x) && isfinite((double)p.y) && isfinite((double)p.z)))
      o->status |= ST_NONFINITE;
    if (out->path > (real)0.5 * o->skin) req = 1;
    o->cap_f[i] = f;
    o->cap_t[i] = t;
  }
  if (o->mix)
    for (int p = 0; p < o->mix->npoly; ++p) mix_poly_step(o, p, &req);
  part* tmp = o->p; o->p = o->q; o->q = tmp;
  if (req) o->rebuild_req = 1;
  /* the drums' turn advances after the step (k_ens_rot_tick) */
  for (int s = 0; s < o->nsys; ++s) {
    if (!o->S[s].rot) continue;
    const real c0 = o->rot_c[s], s0 = o->rot_s[s];
    const real c1 = c0 * o->S[s].rot_cd - s0 * o->S[s].rot_sd;
    const real s1 = s0 * o->S[s].rot_cd + c0 * o->S[s].rot_sd;
    const real m = SQRT(c1 * c1 + s1 * s1);
    o->rot_c[s] = c1 / m;
    o->rot_s[s] = s1 / m;
  }
}

int ens_step(ens_oracle* o, int nsteps) {
  for (int s = 0; s < nsteps; ++s) step_once(o);
  return (int)o->status;
}

void ens_get_state(const ens_oracle* o, double* pos3, double* rad, double* vel3, double* avel3,
                   int* sys, int* pid) {
  for (int i = 0; i < o->n; ++i) {
    const part* a = &o->p[i];
    if (pos3) { pos3[3 * i] = a->pos.x; pos3[3 * i + 1] = a->pos.y; pos3[3 * i + 2] = a->pos.z; }
    if (rad) rad[i] = a->r;
    if (vel3) { vel3[3 * i] = a->vel.x; vel3[3 * i + 1] = a->vel.y; vel3[3 * i + 2] = a->vel.z; }
    if (avel3) { avel3[3 * i] = a->w.x; avel3[3 * i + 1] = a->w.y; avel3[3 * i + 2] = a->w.z; }
    if (sys) sys[i] = a->sys;
    if (pid) pid[i] = a->pid;
  }
}

void ens_get_forces(const ens_oracle* o, double* f3, double* t3) {
  for (int i = 0; i < o->n; ++i) {
    f3[3 * i] = o->cap_f[i].x; f3[3 * i + 1] = o->cap_f[i].y; f3[3 * i + 2] = o->cap_f[i].z;
    t3[3 * i] = o->cap_t[i].x; t3[3 * i + 1] = o->cap_t[i].y; t3[3 * i + 2] = o->cap_t[i].z;
  }
}

int ens_num_rebuilds(const ens_oracle* o) { return o->epoch; }
int ens_status(const ens_oracle* o) { return (int)o->status; }

/* ======================================================== reverse sweep
 * Discrete adjoint of the step for the linear law (no rolling friction)
 * with plane walls: the exact derivative of the forward's arithmetic on the
 * branch each contact took (contact or not, stick or slip, history turned or
 * not), i.e. active-branch derivatives at contact onset and stick/slip
 * switches. */

typedef struct { real kn, kt, b2, mu; } lawbar;

/* Cotangents of contact_law's inputs (n, delta, vrel, vct, xi) and of the
 * law constants, for cotangents Fb (force on a), Tb (torque on a) and Xb
 * (history after the step), linear law. */
static void contact_vjp(const ens_oracle* o, const sysc* S, real mu, v3 n, real delta, real ms,
                        v3 vrel, v3 vct, real arm, v3 x, v3 Fb, v3 Tb, v3 Xb, v3* nb_out,
                        real* deltab_out, v3* vrelb_out, v3* vctb_out, v3* xb_out, lawbar* th) {
  const real dt = o->dt;
  const real kn = S->kn, kt = S->kt;
  /* forward, with the intermediates the reverse needs */
  const real sqn = SQRT(ms * kn), sqt = SQRT(ms * kt);
  const real cn = S->beta2 * sqn, ct = S->beta2 * sqt;
  const real vn = dot(vrel, n);
  const real fn = kn * delta - cn * vn;
  const real fc = fn > 0 ? fn : 0;
  const real p = dot(vct, n);
  const v3 vt = sub(vct, smul(p, n));
  const real xn = dot(x, n);
  const int rot = xn != 0;
  real m0 = 0, m1 = 0, g = 1;
  v3 x1 = x;
  if (rot) {
    m0 = dot(x, x);
    x1 = sub(x, smul(xn, n));
    m1 = dot(x1, x1);
    if (m1 > 0) g = SQRT(m0 / m1);
  }
  const v3 x2 = (rot && m1 > 0) ? mul(x1, g) : x1;
  const v3 x3 = add(x2, mul(vt, dt));
  const v3 ft = sub(mul(x3, -kt), mul(vt, ct));
  const real cap = mu * fc;
  const real f2 = dot(ft, ft);
  const int slip = f2 > cap * cap;
  real fmag = 0, s = 1;
  v3 ftp = ft;
  if (slip) {
    fmag = SQRT(f2);
    s = cap / fmag;
    ftp = mul(ft, s);
  }
  const v3 F = add(mul(n, fn), ftp);
  /* reverse */
  v3 nb = mk(0, 0, 0), vtb = mk(0, 0, 0), xb = mk(0, 0, 0), ftb, x3b;
  real fcb = 0, ctb = 0, ktb = 0, knb = 0, cnb = 0, mub = 0;
  const v3 u = mul(n, -arm);                   /* T = u x F */
  nb = add(nb, mul(cross(F, Tb), -arm));
  const v3 Ft = add(Fb, cross(Tb, u));
  real fnb = dot(Ft, n);                       /* F = n fn + ftp */
  nb = add(nb, mul(Ft, fn));
  v3 ftpb = Ft;
  if (slip) {
    const real ik = (real)-1.0 / kt;           /* x4 = (ftp + vt ct) (-1/kt) */
    const v3 A = add(ftp, mul(vt, ct));
    ftpb = add(ftpb, mul(Xb, ik));
    vtb = add(vtb, mul(Xb, ik * ct));
    ctb += dot(vt, Xb) * ik;
    ktb += dot(A, Xb) / (kt * kt);
    ftb = mul(ftpb, s);                        /* ftp = ft s */
    const real sb = dot(ft, ftpb);
    const real capb = sb / fmag;               /* s = cap / |ft| */
    const real fmagb = -sb * cap / (fmag * fmag);
    ftb = add(ftb, mul(ft, fmagb / fmag));
    mub += capb * fc;
    fcb += capb * mu;
    x3b = mk(0, 0, 0);
  } else {
    ftb = ftpb;
    x3b = Xb;
  }
  x3b = add(x3b, mul(ftb, -kt));               /* ft = x3 (-kt) - vt ct */
  ktb -= dot(x3, ftb);
  ctb -= dot(vt, ftb);
  vtb = add(vtb, mul(ftb, -ct));
  const v3 x2b = x3b;                          /* x3 = x2 + vt dt */
  vtb = add(vtb, mul(x3b, dt));
  if (rot) {
    v3 x1b = x2b;
    if (m1 > 0) {
      x1b = mul(x2b, g);                       /* x2 = x1 sqrt(m0 / m1) */
      const real gb = dot(x1, x2b);
      const real m0b = gb * g / (2 * m0);
      const real m1b = -gb * g / (2 * m1);
      x1b = add(x1b, mul(x1, 2 * m1b));
      xb = add(xb, mul(x, 2 * m0b));
    }
    xb = add(xb, x1b);                         /* x1 = x - xn n */
    const real xnb = -dot(n, x1b);
    nb = add(nb, mul(x1b, -xn));
    xb = add(xb, mul(n, xnb));                 /* xn = x . n */
    nb = add(nb, mul(x, xnb));
  } else {
    xb = x2b;
  }
  if (fn > 0) fnb += fcb;                      /* fc = max(fn, 0) */
  v3 vctb = vtb;                               /* vt = vct - (vct . n) n */
  const real pb = -dot(n, vtb);
  nb = add(nb, mul(vtb, -p));
  vctb = add(vctb, mul(n, pb));
  nb = add(nb, mul(vct, pb));
  knb += fnb * delta;                          /* fn = kn delta - cn vn */
  const real deltab = kn * fnb;
  cnb -= fnb * vn;
  const real vnb = -cn * fnb;
  const v3 vrelb = mul(n, vnb);                /* vn = vrel . n */
  nb = add(nb, mul(vrel, vnb));
  th->b2 += cnb * sqn + ctb * sqt;             /* c = 2 beta sqrt(m* k) */
  knb += cnb * S->beta2 * ms / (2 * sqn);
  ktb += ctb * S->beta2 * ms / (2 * sqt);
  th->kn += knb;
  th->kt += ktb;
  th->mu += mub;
  *nb_out = nb;
  *deltab_out = deltab;
  *vrelb_out = vrelb;
  *vctb_out = vctb;
  *xb_out = xb;
}

/* Cotangents of a pair contact (a = this particle, b = its neighbour, as in
 * step_once) for cotangents Fb, Tb on a's force and torque and Xb on the
 * history after the step.  Adds to a's and b's state cotangents; returns
 * the history cotangent before the step.  Needs the pair in contact. */
typedef struct { v3 x, v, w; } sbar;
static v3 pair_vjp(const ens_oracle* o, const sysc* S, const part* a, const part* b, v3 xi,
                   v3 Fb, v3 Tb, v3 Xb, sbar* ab, sbar* bb, lawbar* th) {
  const real ra = a->r, rb = b->r;
  const v3 rel = sub(a->pos, b->pos);
  const real dist = SQRT(dot(rel, rel));
  const real inv = (real)1.0 / dist;
  const v3 n = mul(rel, inv);
  const real delta = overlap_pair(ra, rb, a->pos, b->pos);
  const real ma = S->dens43pi * ((ra * ra) * ra), mb = S->dens43pi * ((rb * rb) * rb);
  const real ms = (ma * mb) / (ma + mb);
  const v3 ua = mul(n, -ra), ub = mul(n, rb);
  const v3 vca = add(a->vel, cross(a->w, ua));
  const v3 vcb = add(b->vel, cross(b->w, ub));
  v3 nb, vrelb, vctb, xib;
  real deltab;
  contact_vjp(o, S, S->mu, n, delta, ms, sub(a->vel, b->vel), sub(vca, vcb), ra, xi, Fb, Tb, Xb,
              &nb, &deltab, &vrelb, &vctb, &xib, th);
  /* vct = vca - vcb, vca = va + wa x ua, vcb = vb + wb x ub */
  ab->v = add(ab->v, vctb);
  ab->w = add(ab->w, cross(ua, vctb));
  nb = add(nb, mul(cross(vctb, a->w), -ra));
  const v3 vcbb = mul(vctb, -1);
  bb->v = add(bb->v, vcbb);
  bb->w = add(bb->w, cross(ub, vcbb));
  nb = add(nb, mul(cross(vcbb, b->w), rb));
  ab->v = add(ab->v, vrelb);                   /* vrel = va - vb */
  bb->v = sub(bb->v, vrelb);
  real distb = -deltab;                        /* delta = (ra + rb) - dist */
  v3 relb = mul(nb, inv);                      /* n = rel / dist */
  distb -= dot(rel, nb) * inv * inv;
  relb = add(relb, mul(rel, distb / dist));    /* dist = |rel| */
  ab->x = add(ab->x, relb);
  bb->x = sub(bb->x, relb);
  return xib;
}

/* Cotangents of a plane-wall contact of particle a; the wall friction
 * coefficient's cotangent is added to *mu_wb. */
static v3 plane_vjp(const ens_oracle* o, const sysc* S, const wallc* W, const part* a, v3 xi,
                    v3 Fb, v3 Tb, v3 Xb, sbar* ab, lawbar* th, real* mu_wb) {
  const real r = a->r;
  const v3 n = W->a;
  const real delta = overlap_plane(r, W->a, W->r, a->pos);
  const real ma = S->dens43pi * ((r * r) * r);
  const v3 ua = mul(n, -r);
  const v3 vca = add(a->vel, cross(a->w, ua));
  v3 nb, vrelb, vctb, xib;
  real deltab;
  lawbar tw = {0, 0, 0, 0};
  contact_vjp(o, S, S->mu_w, n, delta, ma, a->vel, vca, r, xi, Fb, Tb, Xb, &nb, &deltab, &vrelb,
              &vctb, &xib, &tw);
  th->kn += tw.kn;
  th->kt += tw.kt;
  th->b2 += tw.b2;
  *mu_wb += tw.mu;
  ab->v = add(ab->v, add(vrelb, vctb));        /* vrel = va, vct = va + wa x ua */
  ab->w = add(ab->w, cross(ua, vctb));
  ab->x = add(ab->x, mul(n, -deltab));         /* delta = r - (n . x - d); n is fixed */
  return xib;
}

/* Reverse sweep.  ens_adj_record runs `nsteps` steps from the current state
 * and keeps their tape (the state advances); ens_adj_reverse then
 * propagates the cotangents of the final state (gx_f, gv_f, gw_f: 3 per
 * particle, final memory order) back to the recorded initial state (gx0,
 * gv0, gw0: its memory order) and to the five law constants of every system
 * (gth: nsys x {kn, kt, 2 beta, mu, mu_wall}), and frees the tape.  Linear
 * law, plane walls, no rolling friction; record returns -1 for anything
 * else. */
static void free_tape(ens_oracle* o) {
  for (int s = 0; s < o->ntape; ++s) {
    tstep* t = &o->tape[s];
    free(t->perm); free(t->src); free(t->p); free(t->idx); free(t->cnt); free(t->mask);
    free(t->hist);
  }
  free(o->tape);
  o->tape = NULL;
  o->ntape = 0;
}

int ens_adj_record(ens_oracle* o, int nsteps) {
  const int n = o->n, cap = o->cap;
  const size_t ns = (size_t)cap * n;
  if (o->law != BLAZE_LAW_LINEAR) return -1;
  for (int s = 0; s < o->nsys; ++s)
    if (o->S[s].mu_r > 0 || o->S[s].ntri > 0) return -1;
  for (int w = 0; w < o->nwalls; ++w)
    if (o->W[w].kind != BLAZE_WALL_PLANE) return -1;
  free_tape(o);
  tstep* T = (tstep*)calloc(nsteps, sizeof(tstep));
  o->tape = T;
  o->ntape = nsteps;
  for (int s = 0; s < nsteps; ++s) {
    T[s].perm = (int*)malloc(sizeof(int) * n);
    T[s].src = (int*)malloc(sizeof(int) * ns);
    T[s].p = (part*)malloc(sizeof(part) * n);
    T[s].idx = (uint32_t*)malloc(sizeof(uint32_t) * ns);
    T[s].cnt = (uint32_t*)malloc(sizeof(uint32_t) * n);
    T[s].mask = (uint32_t*)malloc(sizeof(uint32_t) * n);
    T[s].hist = (real*)malloc(sizeof(real) * 3 * ns);
    step_once_rec(o, &T[s]);
  }
  return (int)o->status;
}

int ens_adj_reverse(ens_oracle* o, const double* gx_f, const double* gv_f, const double* gw_f,
                    double* gx0, double* gv0, double* gw0, double* gth) {
  const int n = o->n, cap = o->cap, nsteps = o->ntape;
  const size_t ns = (size_t)cap * n;
  tstep* T = o->tape;
  if (!T) return -1;
  const real dt = o->dt;
  sbar* g = (sbar*)calloc(n, sizeof(sbar));
  sbar* gin = (sbar*)calloc(n, sizeof(sbar));
  v3* gH = (v3*)calloc(ns, sizeof(v3));
  v3* gHin = (v3*)calloc(ns, sizeof(v3));
  v3* gW = (v3*)calloc((size_t)n * WSLOTS, sizeof(v3));
  v3* gWin = (v3*)calloc((size_t)n * WSLOTS, sizeof(v3));
  v3* Fb = (v3*)calloc(n, sizeof(v3));
  v3* Tb = (v3*)calloc(n, sizeof(v3));
  lawbar* th = (lawbar*)calloc(o->nsys, sizeof(lawbar));
  real* muw = (real*)calloc(o->nsys, sizeof(real));
  for (int i = 0; i < n; ++i) {
    g[i].x = mk(gx_f[3 * i], gx_f[3 * i + 1], gx_f[3 * i + 2]);
    g[i].v = mk(gv_f[3 * i], gv_f[3 * i + 1], gv_f[3 * i + 2]);
    g[i].w = mk(gw_f[3 * i], gw_f[3 * i + 1], gw_f[3 * i + 2]);
  }
  int rc = (int)o->status;
  for (int s = nsteps - 1; s >= 0 && rc >= 0; --s) {
    const tstep* t = &T[s];
    const part* P = t->p;
    /* symplectic Euler: v' = v + (f/m + g) dt, x' = x + v' dt, w' = w + t/I dt */
    for (int i = 0; i < n; ++i) {
      const sysc* S = &o->S[P[i].sys];
      const real r = P[i].r;
      const real m = S->dens43pi * ((r * r) * r);
      const real inertia = ((real)0.4 * m) * (r * r);
      const v3 gv = add(g[i].v, mul(g[i].x, dt));
      Fb[i] = mul(gv, dt / m);
      Tb[i] = mul(g[i].w, dt / inertia);
      gin[i].x = g[i].x;
      gin[i].v = gv;
      gin[i].w = g[i].w;
    }
    memset(gHin, 0, sizeof(v3) * ns);
    memset(gWin, 0, sizeof(v3) * (size_t)n * WSLOTS);
    for (int i = 0; i < n && rc >= 0; ++i) {
      const part* a = &P[i];
      const sysc* S = &o->S[a->sys];
      lawbar* tb = &th[a->sys];
      const real ra = a->r;
      for (uint32_t k = 0; k < t->cnt[i]; ++k) {
        const size_t sk = (size_t)k * n + i;
        const part* b = &P[t->idx[sk]];
        const v3 rel = sub(a->pos, b->pos);
        const real sr = ra + b->r;
        const real d2 = dot(rel, rel);
        if (!(d2 < sr * sr) || !(SQRT(d2) > 0)) continue;
        if (!(overlap_pair(ra, b->r, a->pos, b->pos) > 0)) continue;
        const int had = (t->mask[i] >> k) & 1u;
        const v3 xi = had ? mk(t->hist[3 * sk], t->hist[3 * sk + 1], t->hist[3 * sk + 2]) : mk(0, 0, 0);
        const v3 xib = pair_vjp(o, S, a, b, xi, Fb[i], Tb[i], gH[sk], &gin[i], &gin[t->idx[sk]], tb);
        if (had) gHin[sk] = xib;
      }
      int nw = 0;
      for (int w = S->wall0; w < S->wall0 + S->nwall; ++w) {
        v3 nn;
        real d;
        int reg;
        if (!wall_touch(&o->W[w], a->pos, ra, &nn, &d, &reg)) continue;
        int q_old = -1;
        for (int q = 0; q < WSLOTS; ++q)
          if (((a->wmask >> q) & 1u) && a->wid[q] == w) q_old = q;
        const v3 xi = q_old >= 0 ? mk(a->wh[q_old][0], a->wh[q_old][1], a->wh[q_old][2]) : mk(0, 0, 0);
        const v3 Xb = nw < WSLOTS ? gW[(size_t)i * WSLOTS + nw] : mk(0, 0, 0);
        const v3 xib = plane_vjp(o, S, &o->W[w], a, xi, Fb[i], Tb[i], Xb, &gin[i], tb, &muw[a->sys]);
        if (q_old >= 0) gWin[(size_t)i * WSLOTS + q_old] = xib;
        ++nw;
      }
    }
    if (t->rebuilt) {
      /* the step read the re-sorted state: send the cotangents back through
         the permutation and the history carry-over */
      memset(g, 0, sizeof(sbar) * n);
      memset(gH, 0, sizeof(v3) * ns);
      memset(gW, 0, sizeof(v3) * (size_t)n * WSLOTS);
      for (int i = 0; i < n; ++i) {
        const int io = t->perm[i];
        g[io] = gin[i];
        for (int q = 0; q < WSLOTS; ++q) gW[(size_t)io * WSLOTS + q] = gWin[(size_t)i * WSLOTS + q];
        for (uint32_t k = 0; k < t->cnt[i]; ++k) {
          const size_t sk = (size_t)k * n + i;
          if (t->src[sk] >= 0) gH[(size_t)t->src[sk] * n + io] = gHin[sk];
        }
      }
    } else {
      memcpy(g, gin, sizeof(sbar) * n);
      memcpy(gH, gHin, sizeof(v3) * ns);
      memcpy(gW, gWin, sizeof(v3) * (size_t)n * WSLOTS);
    }
  }
  for (int i = 0; i < n; ++i) {
    gx0[3 * i] = g[i].x.x; gx0[3 * i + 1] = g[i].x.y; gx0[3 * i + 2] = g[i].x.z;
    gv0[3 * i] = g[i].v.x; gv0[3 * i + 1] = g[i].v.y; gv0[3 * i + 2] = g[i].v.z;
    gw0[3 * i] = g[i].w.x; gw0[3 * i + 1] = g[i].w.y; gw0[3 * i + 2] = g[i].w.z;
  }
  for (int s = 0; s < o->nsys; ++s) {
    gth[5 * s] = th[s].kn; gth[5 * s + 1] = th[s].kt; gth[5 * s + 2] = th[s].b2;
    gth[5 * s + 3] = th[s].mu; gth[5 * s + 4] = muw[s];
  }
  free_tape(o);
  free(g); free(gin); free(gH); free(gHin); free(gW); free(gWin); free(Fb); free(Tb);
  free(th); free(muw);
  return rc;
}
