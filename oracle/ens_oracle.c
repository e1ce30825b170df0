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
  real r, path;
  int sys, pid;
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
  return o;
}

static void free_tape(ens_oracle* o);
void ens_destroy(ens_oracle* o) {
  if (!o) return;
  free_tape(o);
  free(o->S); free(o->W); free(o->p); free(o->q);
  for (int c = 0; c < 2; ++c) { free(o->idx[c]); free(o->cnt[c]); free(o->mask[c]); free(o->hist[c]); }
  free(o->cstart); free(o->cend); free(o->cap_f); free(o->cap_t); free(o->sys_of);
  free(o->rot_c); free(o->rot_s);
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
    for (int q = 0; q < WSLOTS; ++q) a->wid[q] = -1;
  }
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
  for (int i = 0; i < n; ++i) {
    const part* a = &o->p[i];
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
      int nface = 0, best = -1;
      real best_d = 0;
      for (int w = S->tri0; w < S->tri0 + S->ntri; ++w) {
        v3 nn; real d; int reg;
        if (!wall_touch(&o->W[w], pd, ra, &nn, &d, &reg)) continue;
        if (reg == 0) ++nface;
        else if (best < 0 || d > best_d) { best = w; best_d = d; }
      }
      for (int w = S->tri0; w < S->tri0 + S->ntri; ++w) {
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
