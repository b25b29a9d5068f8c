/*
 * nbc_oracle.c -- FP64 CPU restatement of the reference's clump step.
 *
 * TEST INFRASTRUCTURE ONLY (see nbc_oracle.h).  Every function cites the
 * reference file:line it restates.  Expression grouping follows the
 * reference's source so that results agree to rounding (the reference runs
 * with FMA contraction on the GPU; this file is compiled without FMA).
 */
#include "nbc_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double x, y, z; } d3;
typedef struct { double x, y, z, w; } d4;

/* ---------------------------------------------------------------------------
 * vector algebra of src/type.h
 * ------------------------------------------------------------------------- */
static inline d3 mk3(double x, double y, double z) { d3 v = {x, y, z}; return v; }
static inline d3 add3(d3 a, d3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub3(d3 a, d3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 mul3(double s, d3 u) { return mk3(s * u.x, s * u.y, s * u.z); }
static inline double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross3(d3 a, d3 b) {              /* src/type.h:98-110 */
    double x = a.y * b.z - a.z * b.y;
    double y = a.z * b.x - a.x * b.z;
    double z = a.x * b.y - a.y * b.x;
    return mk3(x, y, z);
}
static inline double length3(d3 v) {                /* src/type.h:112-127 */
    double t = v.x * v.x + v.y * v.y + v.z * v.z;
    return t > 1e-32 ? sqrt(t) : 0.0;
}
static inline d3 norm3(d3 v) {                      /* src/type.h:75-93 */
    double t = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    if (t > 1e-20) return mk3(v.x / t, v.y / t, v.z / t);
    return mk3(0, 0, 0);
}
static inline d4 add4(d4 a, d4 b) { d4 v = {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; return v; }
static inline d4 mul4(double s, d4 u) { d4 v = {s * u.x, s * u.y, s * u.z, s * u.w}; return v; }

/* Quat2DCM (C_nb, world->body), src/type.h:223-236 */
static void quat2dcm(d4 q, double m[3][3]) {
    m[0][0] = q.x * q.x - q.y * q.y - q.z * q.z + q.w * q.w;
    m[1][0] = 2.0 * (q.x * q.y - q.z * q.w);
    m[2][0] = 2.0 * (q.x * q.z + q.y * q.w);
    m[0][1] = 2.0 * (q.x * q.y + q.z * q.w);
    m[1][1] = -q.x * q.x + q.y * q.y - q.z * q.z + q.w * q.w;
    m[2][1] = 2.0 * (q.y * q.z - q.x * q.w);
    m[0][2] = 2.0 * (q.x * q.z - q.y * q.w);
    m[1][2] = 2.0 * (q.y * q.z + q.x * q.w);
    m[2][2] = -q.x * q.x - q.y * q.y + q.z * q.z + q.w * q.w;
}
/* Quat2IvDCM (C_bn, body->world), src/type.h:238-250 */
static void quat2ivdcm(d4 q, double m[3][3]) {
    m[0][0] = q.x * q.x - q.y * q.y - q.z * q.z + q.w * q.w;
    m[1][0] = 2.0 * (q.x * q.y + q.z * q.w);
    m[2][0] = 2.0 * (q.x * q.z - q.y * q.w);
    m[0][1] = 2.0 * (q.x * q.y - q.z * q.w);
    m[1][1] = -q.x * q.x + q.y * q.y - q.z * q.z + q.w * q.w;
    m[2][1] = 2.0 * (q.y * q.z + q.x * q.w);
    m[0][2] = 2.0 * (q.x * q.z + q.y * q.w);
    m[1][2] = 2.0 * (q.y * q.z - q.x * q.w);
    m[2][2] = -q.x * q.x - q.y * q.y + q.z * q.z + q.w * q.w;
}
/* Map, src/type.h:296-305 */
static inline d3 map3(double m[3][3], d3 u) {
    double a = m[0][0] * u.x + m[0][1] * u.y + m[0][2] * u.z;
    double b = m[1][0] * u.x + m[1][1] * u.y + m[1][2] * u.z;
    double c = m[2][0] * u.x + m[2][1] * u.y + m[2][2] * u.z;
    return mk3(a, b, c);
}

#define PI_REF 3.14159265359 /* src/dem_constant.h:14 */

/* ---------------------------------------------------------------------------
 * state
 * ------------------------------------------------------------------------- */
struct nbo_scene {
    /* Parameters (src/dem_parameters.h) */
    int N, K, BL, cellnum;
    int gdim[3];
    double cell[3], icell[3], origin[3], wsize[3], box_lo[3], box_hi[3];
    double dt, E, nu, mu, damping, gravity, beta, cohesion, thresh;
    unsigned update;
    int is_wall, is_intruder, start_step, step, rebuilds, output_interval, count;
    /* subspheres, sorted order */
    int *clump_id, *part_fix;
    d3 *pos, *local, *cum;
    double *mass, *radius;
    /* grid */
    int *part_cel, *part_idx_pre, *cell_beg, *cell_end, *tmp_i;
    int *Ng, *Ni, *Nsum, *Nsum_pre, *Lpa, *Lpb, *Lpb_pre, *Anei, *Aref;
    size_t cap;       /* N * BL / 2 */
    size_t hw;        /* slots ever written (high-water mark) */
    int npairs;
    /* pair force (DEMForce) */
    d3 *Fc, *Tc, *Dv, *Dv_pre, *Dt, *Dt_pre, *Dr, *Dr_pre;
    d3 *CacheFc, *CacheTc, *CacheTc2, *CacheFcn, *CacheCpt;
    /* cube wall: 6 faces x (Dv, Dt, Dr), current and previous */
    int has_cube;
    d3 cube_half, cube_c, cube_v, cube_w;
    d3 *wc_hist[6][3], *wc_hist_pre[6][3];
    /* cylinder wall: 3 regions (bottom cap, top cap, side) */
    int has_cyl;
    double cyl_R, cyl_H;
    d3 cyl_axis, cyl_c, cyl_v, cyl_w;
    d3 *cy_hist[3][3], *cy_hist_pre[3][3];
    d3 *Fw, *Tw;
    /* intruder */
    int intr_shape, intr_motion, intr_wait, intr_state;
    double intr_R, intr_H;
    d3 intr_axis, intr_p, intr_v, intr_w;
    d4 intr_prop;
    d3 *Fi, *Ti, *peneTc, *Fcn_i, *Fct_i, *Tcn_i, *Tct_i, *RVo_i, *RVn_i;
    d3 *pe_Dv, *pe_Dv_pre, *pe_Dt, *pe_Dt_pre, *pe_Dr, *pe_Dr_pre;
    int *LcFlg;
    d3 totFc, totTc, reaction, reaction_t;
    /* sum of all forces */
    d3 *totF, *totT;
    /* clumps */
    d3 *cpos, *cvel, *cw, *cFc, *cTc;
    d4 *cq, *cprop;
    int *mem_order; /* subsphere indices sorted by clump id (stable) */
    int *mem_start; /* [K+1] */
    /* hierarchical grid */
    int levels;
    int* level;            /* per subsphere, sorted order */
    double* lcell;         /* [levels] */
    int (*ldim)[3];        /* [levels] */
    int* loff;             /* [levels] */
    /* sphere-only drivers */
    int sphere;            /* SPH_* bits */
    int* kind;             /* [K] split driver Type per sphere (= clump) */
    d3* scum;              /* [K] CumPos of the sphere drivers */
};
enum { SPH_KIN = 1, SPH_CUBE = 2, SPH_RESET = 4 };

static int g_threads = 1;
void nbo_set_threads(int n) { g_threads = n > 0 ? n : 1; }

static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    if (!p) abort();
    return p;
}

/* LoadParameters damping (src/dem_subsphere_io.cu:143-145) and SetMeshSize
 * (src/dem_subsphere_io.cu:195-230). */
nbo_scene* nbo_create(const nbo_desc* d) {
    nbo_scene* s = (nbo_scene*)xcalloc(1, sizeof(nbo_scene));
    int N = d->N, K = d->K;
    s->N = N; s->K = K; s->BL = d->BL;
    s->dt = d->dt; s->E = d->E; s->nu = d->nu; s->mu = d->mu; s->beta = d->beta;
    s->cohesion = d->cohesion; s->gravity = d->gravity; s->thresh = d->thresh;
    double lnCOR = log(d->e_rest);
    s->damping = 2.0 * sqrt(5.0 / 6.0) * lnCOR / sqrt(lnCOR * lnCOR + PI_REF * PI_REF);
    s->is_wall = d->is_wall; s->is_intruder = d->is_intruder;
    s->start_step = d->start_step; s->step = d->start_step;
    s->output_interval = d->output_interval > 0 ? d->output_interval : 1;

    double rmax = 0.0;
    for (int i = 0; i < N; i++) if (d->radius[i] > rmax) rmax = d->radius[i];
    double mesh = 3.0 * rmax;
    s->levels = d->levels > 1 ? d->levels : 1;
    for (int a = 0; a < 3; a++) {
        s->cell[a] = mesh;
        s->icell[a] = 1.0 / mesh;
        s->origin[a] = d->world_origin[a] - s->cell[a];
        s->wsize[a] = d->world_size[a] + 2 * s->cell[a];
        s->gdim[a] = (int)(unsigned)ceil(s->wsize[a] / s->cell[a]);
        s->box_lo[a] = d->box_lo[a];
        s->box_hi[a] = d->box_hi[a];
    }
    s->cellnum = s->gdim[0] * s->gdim[1] * s->gdim[2];
    if (s->levels > 1) {
        s->lcell = (double*)xcalloc(s->levels, sizeof(double));
        s->ldim = xcalloc(s->levels, sizeof(int[3]));
        s->loff = (int*)xcalloc(s->levels, sizeof(int));
        int off = 0;
        for (int l = 0; l < s->levels; l++) {
            s->lcell[l] = d->level_cell[l];
            for (int a = 0; a < 3; a++)
                s->ldim[l][a] = (int)ceil(s->wsize[a] / s->lcell[l]);
            s->loff[l] = off;
            off += s->ldim[l][0] * s->ldim[l][1] * s->ldim[l][2];
        }
        s->cellnum = off + 1; /* last bucket = out of box */
        s->level = (int*)xcalloc(N, sizeof(int));
        for (int i = 0; i < N; i++) s->level[i] = d->level[i];
    }

    s->clump_id = (int*)xcalloc(N, sizeof(int));
    s->part_fix = (int*)xcalloc(N, sizeof(int));
    s->pos = (d3*)xcalloc(N, sizeof(d3));
    s->local = (d3*)xcalloc(N, sizeof(d3));
    s->cum = (d3*)xcalloc(N, sizeof(d3));
    s->mass = (double*)xcalloc(N, sizeof(double));
    s->radius = (double*)xcalloc(N, sizeof(double));
    for (int i = 0; i < N; i++) {
        s->clump_id[i] = d->clump_id[i];
        s->part_fix[i] = i; /* GetParticleFixIndex_cuk, src/dem_grid.cu:204-210 */
        s->pos[i] = mk3(d->pos[3 * i], d->pos[3 * i + 1], d->pos[3 * i + 2]);
        s->local[i] = mk3(d->local[3 * i], d->local[3 * i + 1], d->local[3 * i + 2]);
        s->mass[i] = d->mass[i];
        s->radius[i] = d->radius[i];
    }
    s->cap = (size_t)N * (size_t)(s->BL / 2);
    size_t rows = (size_t)N * (size_t)s->BL;
    s->part_cel = (int*)xcalloc(N, sizeof(int));
    s->part_idx_pre = (int*)xcalloc(N, sizeof(int));
    s->tmp_i = (int*)xcalloc(N, sizeof(int));
    s->cell_beg = (int*)xcalloc(s->cellnum, sizeof(int));
    s->cell_end = (int*)xcalloc(s->cellnum, sizeof(int));
    s->Ng = (int*)xcalloc(N, sizeof(int));
    s->Ni = (int*)xcalloc(N, sizeof(int));
    s->Nsum = (int*)xcalloc(N, sizeof(int));
    s->Nsum_pre = (int*)xcalloc(N, sizeof(int));
    s->Lpa = (int*)xcalloc(s->cap, sizeof(int));
    s->Lpb = (int*)xcalloc(s->cap, sizeof(int));
    s->Lpb_pre = (int*)xcalloc(s->cap, sizeof(int));
    memset(s->Lpb, 0xFF, s->cap * sizeof(int));
    memset(s->Lpb_pre, 0xFF, s->cap * sizeof(int));
    s->Anei = (int*)xcalloc(rows, sizeof(int));
    s->Aref = (int*)xcalloc(rows, sizeof(int));
    s->Fc = (d3*)xcalloc(N, sizeof(d3));
    s->Tc = (d3*)xcalloc(N, sizeof(d3));
    s->Dv = (d3*)xcalloc(s->cap, sizeof(d3));
    s->Dv_pre = (d3*)xcalloc(s->cap, sizeof(d3));
    s->Dt = (d3*)xcalloc(s->cap, sizeof(d3));
    s->Dt_pre = (d3*)xcalloc(s->cap, sizeof(d3));
    s->Dr = (d3*)xcalloc(s->cap, sizeof(d3));
    s->Dr_pre = (d3*)xcalloc(s->cap, sizeof(d3));
    s->CacheFc = (d3*)xcalloc(s->cap, sizeof(d3));
    s->CacheTc = (d3*)xcalloc(s->cap, sizeof(d3));
    s->CacheTc2 = (d3*)xcalloc(s->cap, sizeof(d3));
    s->CacheFcn = (d3*)xcalloc(s->cap, sizeof(d3));
    s->CacheCpt = (d3*)xcalloc(s->cap, sizeof(d3));

    s->has_cube = d->has_cube;
    s->cube_half = mk3(d->cube_half[0], d->cube_half[1], d->cube_half[2]);
    s->cube_c = mk3(d->cube_centre[0], d->cube_centre[1], d->cube_centre[2]);
    s->cube_v = mk3(d->cube_vel[0], d->cube_vel[1], d->cube_vel[2]);
    s->cube_w = mk3(d->cube_angvel[0], d->cube_angvel[1], d->cube_angvel[2]);
    for (int f = 0; f < 6; f++)
        for (int h = 0; h < 3; h++) {
            s->wc_hist[f][h] = (d3*)xcalloc(N, sizeof(d3));
            s->wc_hist_pre[f][h] = (d3*)xcalloc(N, sizeof(d3));
        }
    s->has_cyl = d->has_cyl;
    s->cyl_R = d->cyl_radius; s->cyl_H = d->cyl_half_height;
    s->cyl_axis = mk3(d->cyl_axis[0], d->cyl_axis[1], d->cyl_axis[2]);
    s->cyl_c = mk3(d->cyl_centre[0], d->cyl_centre[1], d->cyl_centre[2]);
    s->cyl_v = mk3(d->cyl_vel[0], d->cyl_vel[1], d->cyl_vel[2]);
    s->cyl_w = mk3(d->cyl_angvel[0], d->cyl_angvel[1], d->cyl_angvel[2]);
    for (int f = 0; f < 3; f++)
        for (int h = 0; h < 3; h++) {
            s->cy_hist[f][h] = (d3*)xcalloc(N, sizeof(d3));
            s->cy_hist_pre[f][h] = (d3*)xcalloc(N, sizeof(d3));
        }
    s->Fw = (d3*)xcalloc(N, sizeof(d3));
    s->Tw = (d3*)xcalloc(N, sizeof(d3));

    s->intr_shape = d->intr_shape; s->intr_motion = d->intr_motion; s->intr_wait = d->intr_wait;
    s->intr_state = 0;
    s->intr_R = d->intr_radius; s->intr_H = d->intr_half_height;
    s->intr_axis = mk3(d->intr_axis[0], d->intr_axis[1], d->intr_axis[2]);
    s->intr_p = mk3(d->intr_pos[0], d->intr_pos[1], d->intr_pos[2]);
    s->intr_v = mk3(d->intr_vel[0], d->intr_vel[1], d->intr_vel[2]);
    s->intr_w = mk3(d->intr_angvel[0], d->intr_angvel[1], d->intr_angvel[2]);
    s->intr_prop.x = d->intr_prop[0]; s->intr_prop.y = d->intr_prop[1];
    s->intr_prop.z = d->intr_prop[2]; s->intr_prop.w = d->intr_prop[3];
    s->Fi = (d3*)xcalloc(N, sizeof(d3));
    s->Ti = (d3*)xcalloc(N, sizeof(d3));
    s->peneTc = (d3*)xcalloc(N, sizeof(d3));
    s->Fcn_i = (d3*)xcalloc(N, sizeof(d3));
    s->Fct_i = (d3*)xcalloc(N, sizeof(d3));
    s->Tcn_i = (d3*)xcalloc(N, sizeof(d3));
    s->Tct_i = (d3*)xcalloc(N, sizeof(d3));
    s->RVo_i = (d3*)xcalloc(N, sizeof(d3));
    s->RVn_i = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dv = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dv_pre = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dt = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dt_pre = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dr = (d3*)xcalloc(N, sizeof(d3));
    s->pe_Dr_pre = (d3*)xcalloc(N, sizeof(d3));
    s->LcFlg = (int*)xcalloc(N, sizeof(int));
    s->totF = (d3*)xcalloc(N, sizeof(d3));
    s->totT = (d3*)xcalloc(N, sizeof(d3));

    s->cpos = (d3*)xcalloc(K, sizeof(d3));
    s->cvel = (d3*)xcalloc(K, sizeof(d3));
    s->cw = (d3*)xcalloc(K, sizeof(d3));
    s->cFc = (d3*)xcalloc(K, sizeof(d3));
    s->cTc = (d3*)xcalloc(K, sizeof(d3));
    s->cq = (d4*)xcalloc(K, sizeof(d4));
    s->cprop = (d4*)xcalloc(K, sizeof(d4));
    for (int k = 0; k < K; k++) {
        s->cpos[k] = mk3(d->cpos[3 * k], d->cpos[3 * k + 1], d->cpos[3 * k + 2]);
        s->cvel[k] = mk3(d->cvel[3 * k], d->cvel[3 * k + 1], d->cvel[3 * k + 2]);
        s->cw[k] = mk3(d->cangvel[3 * k], d->cangvel[3 * k + 1], d->cangvel[3 * k + 2]);
        d4 q = {d->cquat[4 * k], d->cquat[4 * k + 1], d->cquat[4 * k + 2], d->cquat[4 * k + 3]};
        d4 p = {d->cprop[4 * k], d->cprop[4 * k + 1], d->cprop[4 * k + 2], d->cprop[4 * k + 3]};
        s->cq[k] = q;
        s->cprop[k] = p;
    }
    s->mem_order = (int*)xcalloc(N, sizeof(int));
    s->mem_start = (int*)xcalloc(K + 1, sizeof(int));
    s->sphere = d->sphere_mode;
    if (s->sphere) s->scum = (d3*)xcalloc(K, sizeof(d3));
    if (d->body_kind) {
        s->kind = (int*)xcalloc(K, sizeof(int));
        memcpy(s->kind, d->body_kind, K * sizeof(int));
    }
    return s;
}

void nbo_destroy(nbo_scene* s) {
    if (!s) return;
    void* ptrs[] = {s->clump_id, s->part_fix, s->pos, s->local, s->cum, s->mass, s->radius,
                    s->part_cel, s->part_idx_pre, s->cell_beg, s->cell_end, s->tmp_i, s->Ng,
                    s->Ni, s->Nsum, s->Nsum_pre, s->Lpa, s->Lpb, s->Lpb_pre, s->Anei, s->Aref,
                    s->Fc, s->Tc, s->Dv, s->Dv_pre, s->Dt, s->Dt_pre, s->Dr, s->Dr_pre,
                    s->CacheFc, s->CacheTc, s->CacheTc2, s->CacheFcn, s->CacheCpt, s->Fw, s->Tw,
                    s->Fi, s->Ti, s->peneTc, s->Fcn_i, s->Fct_i, s->Tcn_i, s->Tct_i, s->RVo_i,
                    s->RVn_i, s->pe_Dv, s->pe_Dv_pre, s->pe_Dt, s->pe_Dt_pre, s->pe_Dr,
                    s->pe_Dr_pre, s->LcFlg, s->totF, s->totT, s->cpos, s->cvel, s->cw, s->cFc,
                    s->cTc, s->cq, s->cprop, s->mem_order, s->mem_start, s->level, s->lcell,
                    s->ldim, s->loff, s->kind, s->scum};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    for (int f = 0; f < 6; f++)
        for (int h = 0; h < 3; h++) { free(s->wc_hist[f][h]); free(s->wc_hist_pre[f][h]); }
    for (int f = 0; f < 3; f++)
        for (int h = 0; h < 3; h++) { free(s->cy_hist[f][h]); free(s->cy_hist_pre[f][h]); }
    free(s);
}

/* ---------------------------------------------------------------------------
 * clump kinematics
 * ------------------------------------------------------------------------- */

/* Integrate_Before_clump_cuk + Attitude_clump_cuk,
 * src/dem_integrate_clumpsphere.cu:3-90 */
static void clump_integrate_before(nbo_scene* s) {
    double Dt = s->dt;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->K; i++) {
        d4 P = s->cprop[i];
        d3 F = s->cFc[i], T = s->cTc[i];
        F = mul3(1.0 / P.w, F);
        F.z = F.z + s->gravity;
        T.x = (1.0 / P.x) * T.x;
        T.y = (1.0 / P.y) * T.y;
        T.z = (1.0 / P.z) * T.z;
        d3 dist = add3(mul3(Dt, s->cvel[i]), mul3(0.5 * Dt * Dt, F));
        s->cpos[i] = add3(s->cpos[i], dist);
        s->cvel[i] = add3(s->cvel[i], mul3(0.5 * Dt, F));
        s->cw[i] = add3(s->cw[i], mul3(0.5 * Dt, T));
    }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->K; i++) {
        d4 P = s->cprop[i];
        d3 W = s->cw[i], T = s->cTc[i];
        T.x = (1.0 / P.x) * T.x;
        T.y = (1.0 / P.y) * T.y;
        T.z = (1.0 / P.z) * T.z;
        d4 q = s->cq[i], qd, qdd;
        double m[3][3];
        quat2dcm(q, m);
        d3 Wb = map3(m, W), Wdb = map3(m, T);
        qd.x = 0.50 * (Wb.x * q.w - Wb.y * q.z + Wb.z * q.y);
        qd.y = 0.50 * (Wb.x * q.z + Wb.y * q.w - Wb.z * q.x);
        qd.z = 0.50 * (-Wb.x * q.y + Wb.y * q.x + Wb.z * q.w);
        qd.w = 0.50 * (-Wb.x * q.x - Wb.y * q.y - Wb.z * q.z);
        qdd.x = (Wdb.x * q.w - Wdb.y * q.z + Wdb.z * q.y) * 0.50 +
                (Wb.x * qd.w - Wb.y * qd.z + Wb.z * qd.y) * 0.50;
        qdd.y = (Wdb.x * q.z + Wdb.y * q.w - Wdb.z * q.x) * 0.50 +
                (Wb.x * qd.z + Wb.y * qd.w - Wb.z * qd.x) * 0.50;
        qdd.z = (-Wdb.x * q.y + Wdb.y * q.x + Wdb.z * q.w) * 0.50 +
                (-Wb.x * qd.y + Wb.y * qd.x + Wb.z * qd.w) * 0.50;
        qdd.w = (-Wdb.x * q.x - Wdb.y * q.y - Wdb.z * q.z) * 0.50 +
                (-Wb.x * qd.x - Wb.y * qd.y - Wb.z * qd.z) * 0.50;
        q = add4(add4(q, mul4(Dt, qd)), mul4(0.5 * Dt * Dt, qdd));
        double nrm = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        s->cq[i] = mul4(1.0 / nrm, q);
    }
}

/* Integrate_After_clump_cuk, src/dem_integrate_clumpsphere.cu:110-141 */
static void clump_integrate_after(nbo_scene* s) {
    double Dt = s->dt;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->K; i++) {
        d4 P = s->cprop[i];
        d3 F = s->cFc[i], T = s->cTc[i];
        F = mul3(1.0 / P.w, F);
        F.z = F.z + s->gravity;
        T.x = (1.0 / P.x) * T.x;
        T.y = (1.0 / P.y) * T.y;
        T.z = (1.0 / P.z) * T.z;
        s->cvel[i] = add3(s->cvel[i], mul3(0.5 * Dt, F));
        s->cw[i] = add3(s->cw[i], mul3(0.5 * Dt, T));
    }
}

/* The sphere drivers' integrator, one sphere per clump (sphere i of the
 * sorted order is clump c = clump_id[i], LocalPos = 0):
 * Integrate_Before_cuk + Attitude_cuk (src/dem_integrate.cu:3-100): the
 * first half-kick and the attitude from the contact and wall force and
 * torque only, the displacement accumulated in CumPos.  The split driver
 * (src/dem_integrate_withglue.cu:3-110) is called with the original index
 * where its first half-kick expects Type (src/dem_simulation_split.cu:84-85):
 * its kick and move go by original index (0 free with the 0.1 r rebuild
 * test, 1 driven at (-0.2 y, -0.2 x, 0), 2 and above still), its attitude
 * by Type (turns only for Type 0). */
static void sphere_quat(nbo_scene* s, int c, d3 W, d3 T) {
    double Dt = s->dt;
    d4 q = s->cq[c], qd, qdd;
    double m[3][3];
    quat2dcm(q, m);
    d3 Wb = map3(m, W), Wdb = map3(m, T);
    qd.x = 0.50 * (Wb.x * q.w - Wb.y * q.z + Wb.z * q.y);
    qd.y = 0.50 * (Wb.x * q.z + Wb.y * q.w - Wb.z * q.x);
    qd.z = 0.50 * (-Wb.x * q.y + Wb.y * q.x + Wb.z * q.w);
    qd.w = 0.50 * (-Wb.x * q.x - Wb.y * q.y - Wb.z * q.z);
    qdd.x = (Wdb.x * q.w - Wdb.y * q.z + Wdb.z * q.y) * 0.50 + (Wb.x * qd.w - Wb.y * qd.z + Wb.z * qd.y) * 0.50;
    qdd.y = (Wdb.x * q.z + Wdb.y * q.w - Wdb.z * q.x) * 0.50 + (Wb.x * qd.z + Wb.y * qd.w - Wb.z * qd.x) * 0.50;
    qdd.z = (-Wdb.x * q.y + Wdb.y * q.x + Wdb.z * q.w) * 0.50 + (-Wb.x * qd.y + Wb.y * qd.x + Wb.z * qd.w) * 0.50;
    qdd.w = (-Wdb.x * q.x - Wdb.y * q.y - Wdb.z * q.z) * 0.50 + (-Wb.x * qd.x - Wb.y * qd.y - Wb.z * qd.z) * 0.50;
    q = add4(add4(q, mul4(Dt, qd)), mul4(0.5 * Dt * Dt, qdd));
    double nrm = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    s->cq[c] = mul4(1.0 / nrm, q);
}

static d3 scale_inertia(d4 P, d3 T) {
    T.x = (1.0 / P.x) * T.x;
    T.y = (1.0 / P.y) * T.y;
    T.z = (1.0 / P.z) * T.z;
    return T;
}

static void sphere_integrate_before(nbo_scene* s) {
    double Dt = s->dt;
    int flag = 0;
    for (int i = 0; i < s->N; i++) {
        int c = s->clump_id[i];
        int kb = s->kind ? (c < 3 ? c : 3) : 0;
        d4 P = s->cprop[c];
        if (kb == 0) {
            d3 F = add3(s->Fc[i], s->Fw[i]);
            d3 T = scale_inertia(P, add3(s->Tc[i], s->Tw[i]));
            F = mul3(1.0 / P.w, F);
            F.z = F.z + s->gravity;
            d3 dist = add3(mul3(Dt, s->cvel[c]), mul3(0.5 * Dt * Dt, F));
            s->scum[c] = add3(s->scum[c], dist);
            s->cpos[c] = add3(s->cpos[c], dist);
            s->cvel[c] = add3(s->cvel[c], mul3(0.5 * Dt, F));
            s->cw[c] = add3(s->cw[c], mul3(0.5 * Dt, T));
            double thr = s->kind ? 0.10 * s->radius[i] : s->thresh;
            if (length3(s->scum[c]) > thr) flag = 1;
        } else if (kb == 1) {
            d3 p = s->cpos[c];
            d3 v = mk3(-0.2 * p.y, -0.2 * p.x, 0.0);
            d3 dist = mul3(Dt, v);
            s->scum[c] = add3(s->scum[c], dist);
            s->cpos[c] = add3(p, dist);
            s->cvel[c] = v;
        }
        s->pos[i] = s->cpos[c];
    }
    if (flag && s->update == 0) s->update = 1;
    for (int i = 0; i < s->N; i++) {
        int c = s->clump_id[i];
        if (s->kind && s->kind[c] != 0) continue;
        sphere_quat(s, c, s->cw[c], scale_inertia(s->cprop[c], add3(s->Tc[i], s->Tw[i])));
    }
}

/* Integrate_After_cuk (src/dem_integrate.cu:104-146; the split driver's only
 * for Type 0, src/dem_integrate_withglue.cu:136-160) */
static void sphere_integrate_after(nbo_scene* s) {
    double Dt = s->dt;
    for (int i = 0; i < s->N; i++) {
        int c = s->clump_id[i];
        if (s->kind && s->kind[c] != 0) continue;
        d4 P = s->cprop[c];
        d3 F = add3(add3(s->Fc[i], s->Fw[i]), s->Fi[i]);
        d3 T = scale_inertia(P, add3(add3(s->Tc[i], s->Tw[i]), s->Ti[i]));
        F = mul3(1.0 / P.w, F);
        F.z = F.z + s->gravity;
        s->cvel[c] = add3(s->cvel[c], mul3(0.5 * Dt, F));
        s->cw[c] = add3(s->cw[c], mul3(0.5 * Dt, T));
    }
}

/* UpdatePos_cuk, src/dem_clump.cu:113-138 */
static void update_pos(nbo_scene* s) {
    int flag = 0;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(| : flag)
    for (int i = 0; i < s->N; i++) {
        int c = s->clump_id[i];
        double m[3][3];
        quat2ivdcm(s->cq[c], m);
        d3 arm = map3(m, s->local[i]);
        d3 up = add3(s->cpos[c], arm);
        d3 cum = sub3(add3(s->cum[i], up), s->pos[i]);
        if (length3(cum) > s->thresh) flag = 1;
        s->cum[i] = cum;
        s->pos[i] = up;
    }
    if (flag && s->update == 0) s->update = 1;
}

/* ---------------------------------------------------------------------------
 * broad phase, single level (src/dem_grid.cu)
 * ------------------------------------------------------------------------- */

/* GetParticleCellIndex_cuk, src/dem_grid.cu:155-202 */
static void cell_index(nbo_scene* s) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->N; i++) {
        d3 p = s->pos[i];
        s->part_idx_pre[i] = i;
        if (p.z >= s->box_hi[2] || p.y >= s->box_hi[1] || p.x >= s->box_hi[0] ||
            p.z < s->box_lo[2] || p.y < s->box_lo[1] || p.x < s->box_lo[0]) {
            s->part_cel[i] = s->cellnum - 1;
            continue;
        }
        int cx = (int)floor((p.x - s->origin[0]) / s->cell[0]);
        int cy = (int)floor((p.y - s->origin[1]) / s->cell[1]);
        int cz = (int)floor((p.z - s->origin[2]) / s->cell[2]);
        cx = cx < 0 ? 0 : (cx > s->gdim[0] - 1 ? s->gdim[0] - 1 : cx);
        cy = cy < 0 ? 0 : (cy > s->gdim[1] - 1 ? s->gdim[1] - 1 : cy);
        cz = cz < 0 ? 0 : (cz > s->gdim[2] - 1 ? s->gdim[2] - 1 : cz);
        int idx = cz * s->gdim[1] * s->gdim[0] + cy * s->gdim[0] + cx;
        if (idx < 0) idx = 0;
        if (idx >= s->cellnum) idx = s->cellnum - 1;
        s->part_cel[i] = idx;
    }
}

/* Hierarchical hash, GetParticleCellIndex_hGrid_cuk (src/dem_hgrid.cu:205-242),
 * with the out-of-box bucket kept inside the cell table (cellnum-1). */
static void cell_index_hgrid(nbo_scene* s) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->N; i++) {
        d3 p = s->pos[i];
        s->part_idx_pre[i] = i;
        if (p.z > s->box_hi[2] || p.y > s->box_hi[1] || p.x > s->box_hi[0] ||
            p.z < s->box_lo[2] || p.y < s->box_lo[1] || p.x < s->box_lo[0]) {
            s->part_cel[i] = s->cellnum - 1;
            continue;
        }
        int t = s->level[i];
        double c = s->lcell[t];
        int cx = (int)floor((p.x - s->origin[0]) / c);
        int cy = (int)floor((p.y - s->origin[1]) / c);
        int cz = (int)floor((p.z - s->origin[2]) / c);
        int* n = s->ldim[t];
        cx = cx < 0 ? 0 : (cx > n[0] - 1 ? n[0] - 1 : cx);
        cy = cy < 0 ? 0 : (cy > n[1] - 1 ? n[1] - 1 : cy);
        cz = cz < 0 ? 0 : (cz > n[2] - 1 ? n[2] - 1 : cz);
        s->part_cel[i] = s->loff[t] + (cz * n[1] * n[0] + cy * n[0] + cx);
    }
}

/* SortParticleByCellIndex (src/dem_grid.cu:278-305): CUB's radix sort is
 * stable, so a stable counting sort by cell gives the same permutation. */
static void sort_by_cell(nbo_scene* s) {
    int C = s->cellnum, N = s->N;
    int* cnt = (int*)xcalloc((size_t)C + 1, sizeof(int));
    for (int i = 0; i < N; i++) cnt[s->part_cel[i] + 1]++;
    for (int c = 0; c < C; c++) cnt[c + 1] += cnt[c];
    int* keys = (int*)xcalloc(N, sizeof(int));
    int* perm = (int*)xcalloc(N, sizeof(int));
    int* fix = (int*)xcalloc(N, sizeof(int));
    for (int i = 0; i < N; i++) {
        int dst = cnt[s->part_cel[i]]++;
        keys[dst] = s->part_cel[i];
        perm[dst] = s->part_idx_pre[i];
        fix[dst] = s->part_fix[i];
    }
    memcpy(s->part_cel, keys, N * sizeof(int));
    memcpy(s->part_idx_pre, perm, N * sizeof(int));
    memcpy(s->part_fix, fix, N * sizeof(int));
    free(cnt); free(keys); free(perm); free(fix);
}

/* FindBegEndInCell_cuk, src/dem_grid.cu:105-153 */
static void find_beg_end(nbo_scene* s) {
    for (int c = 0; c < s->cellnum; c++) { s->cell_beg[c] = -1; s->cell_end[c] = -1; }
    for (int i = 0; i < s->N; i++) {
        int c = s->part_cel[i];
        if (c < 0 || c >= s->cellnum) continue;
        if (i == 0 || c != s->part_cel[i - 1]) {
            s->cell_beg[c] = i;
            if (i > 0) {
                int pc = s->part_cel[i - 1];
                if (pc >= 0 && pc < s->cellnum) s->cell_end[pc] = i;
            }
        }
        if (i == s->N - 1) s->cell_end[c] = i + 1;
    }
}

/* SortArray_*_cuk, src/dem_grid.cu:336-437: gather by part_idx_pre. */
static void gather_d3(nbo_scene* s, d3* a) {
    d3* t = (d3*)xcalloc(s->N, sizeof(d3));
    memcpy(t, a, s->N * sizeof(d3));
    for (int i = 0; i < s->N; i++) a[i] = t[s->part_idx_pre[i]];
    free(t);
}
static void gather_d(nbo_scene* s, double* a) {
    double* t = (double*)xcalloc(s->N, sizeof(double));
    memcpy(t, a, s->N * sizeof(double));
    for (int i = 0; i < s->N; i++) a[i] = t[s->part_idx_pre[i]];
    free(t);
}
static void gather_i(nbo_scene* s, int* a) {
    int* t = (int*)xcalloc(s->N, sizeof(int));
    memcpy(t, a, s->N * sizeof(int));
    for (int i = 0; i < s->N; i++) a[i] = t[s->part_idx_pre[i]];
    free(t);
}

static inline int* row(int* base, int BL, int i) { return base + (size_t)i * BL; }

/* CreateAnei_cuk, src/dem_grid.cu:466-552.  Returns 1 on row overflow. */
static int create_anei(nbo_scene* s) {
    int ovf = 0, BL = s->BL;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256) reduction(| : ovf)
    for (int index = 0; index < s->N; index++) {
        if (s->part_cel[index] == s->cellnum - 1) continue;
        d3 pi = s->pos[index];
        double ri = s->radius[index];
        int cx0 = (int)floor((pi.x - s->origin[0]) * s->icell[0]);
        int cy0 = (int)floor((pi.y - s->origin[1]) * s->icell[1]);
        int cz0 = (int)floor((pi.z - s->origin[2]) * s->icell[2]);
        int* ra = row(s->Anei, BL, index);
        for (int cz = -1; cz <= 1; cz++)
            for (int cy = -1; cy <= 1; cy++)
                for (int cx = -1; cx <= 1; cx++) {
                    int x = cx0 + cx, y = cy0 + cy, z = cz0 + cz;
                    if (x < 0 || x >= s->gdim[0] || y < 0 || y >= s->gdim[1] || z < 0 ||
                        z >= s->gdim[2])
                        continue;
                    int c = (z * s->gdim[1] + y) * s->gdim[0] + x;
                    int start = s->cell_beg[c];
                    if (start == -1) continue;
                    int end = s->cell_end[c];
                    for (int j = start; j < end; j++) {
                        if (j == index) continue;
                        d3 pj = s->pos[j];
                        double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                        double d2 = dx * dx + dy * dy + dz * dz;
                        double lim = 1.50 * (ri + s->radius[j]);
                        if (d2 < lim * lim) {
                            if (index < j) {
                                int cnt = s->Ng[index];
                                if (cnt < BL / 2) { ra[cnt] = j; s->Ng[index] = cnt + 1; }
                                else ovf = 1;
                            } else {
                                int cnt = s->Ni[index];
                                if (cnt < BL / 2) { ra[BL - 1 - cnt] = j; s->Ni[index] = cnt + 1; }
                                else ovf = 1;
                            }
                        }
                    }
                }
    }
    return ovf;
}

/* Hierarchical neighbour search, CreateAnei_hGrid_cuk
 * (src/dem_hgrid_contlist.cu:57-161): own level and every coarser level;
 * same-level pairs go by index, cross-level pairs are owned by the coarser
 * (larger) subsphere.  The cross-level entries of a row are sorted by the
 * finer partner's index afterwards so the list is deterministic (the
 * reference claims those slots with atomicAdd, in no fixed order). */
static int create_anei_hgrid(nbo_scene* s) {
    int ovf = 0, BL = s->BL, N = s->N;
    int* cross_cnt = (int*)xcalloc(N, sizeof(int));
    for (int index = 0; index < N; index++) {
        if (s->part_cel[index] == s->cellnum - 1) continue;
        int my = s->level[index];
        d3 pi = s->pos[index];
        double ri = s->radius[index];
        int* ra = row(s->Anei, BL, index);
        for (int t = my; t >= 0; t--) {
            double c = s->lcell[t];
            int* n = s->ldim[t];
            int cx0 = (int)floor((pi.x - s->origin[0]) / c);
            int cy0 = (int)floor((pi.y - s->origin[1]) / c);
            int cz0 = (int)floor((pi.z - s->origin[2]) / c);
            for (int cz = -1; cz <= 1; cz++)
                for (int cy = -1; cy <= 1; cy++)
                    for (int cx = -1; cx <= 1; cx++) {
                        int x = cx0 + cx, y = cy0 + cy, z = cz0 + cz;
                        if (x < 0 || x >= n[0] || y < 0 || y >= n[1] || z < 0 || z >= n[2]) continue;
                        int cell = s->loff[t] + (z * n[1] * n[0] + y * n[0] + x);
                        int start = s->cell_beg[cell];
                        if (start == -1) continue;
                        for (int j = start; j < s->cell_end[cell]; j++) {
                            if (j == index) continue;
                            d3 pj = s->pos[j];
                            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                            double d2 = dx * dx + dy * dy + dz * dz;
                            double lim = 1.5 * (ri + s->radius[j]);
                            if (!(d2 < lim * lim)) continue;
                            if (t == my) {
                                if (index < j) {
                                    if (s->Ng[index] < BL / 2) ra[s->Ng[index]++] = j; else ovf = 1;
                                } else {
                                    if (s->Ni[index] < BL / 2) ra[BL - 1 - s->Ni[index]++] = j; else ovf = 1;
                                }
                            } else {
                                if (s->Ni[index] < BL / 2) ra[BL - 1 - s->Ni[index]++] = j; else ovf = 1;
                                cross_cnt[j]++;
                            }
                        }
                    }
        }
    }
    /* second pass: cross-level entries appended to the coarse row in
     * ascending order of the fine partner */
    for (int index = 0; index < N; index++) {
        int* ra = row(s->Anei, BL, index);
        for (int k = 0; k < s->Ni[index]; k++) {
            int j = ra[BL - 1 - k];
            if (s->level[j] < s->level[index]) {
                if (s->Ng[j] < BL / 2) row(s->Anei, BL, j)[s->Ng[j]++] = index; else ovf = 1;
            }
        }
    }
    free(cross_cnt);
    return ovf;
}

/* CreateContList_cuk, src/dem_grid.cu:561-601 */
static void create_cont_list(nbo_scene* s) {
    int BL = s->BL;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256)
    for (int i = 0; i < s->N; i++) {
        int* ra = row(s->Anei, BL, i);
        int* rr = row(s->Aref, BL, i);
        for (int g = 0; g < s->Ng[i]; g++) {
            int nl = (i == 0) ? g : s->Nsum[i - 1] + g;
            rr[g] = nl;
            int j = ra[g];
            s->Lpa[nl] = i;
            s->Lpb[nl] = j;
            int* ra2 = row(s->Anei, BL, j);
            for (int k = 0; k < s->Ni[j]; k++)
                if (i == ra2[BL - 1 - k]) row(s->Aref, BL, j)[BL - 1 - k] = nl;
        }
    }
}

/* InheritContHistory_cuk, src/dem_grid.cu:603-647.  Writes into `dv` etc.
 * (the caller's *_pre buffers, see create_list_all). */
static void inherit_history(nbo_scene* s, d3* dv, d3* dv_old, d3* dt, d3* dt_old, d3* dr,
                            d3* dr_old) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int nl = 0; nl < s->npairs; nl++) {
        int i = s->Lpa[nl], j = s->Lpb[nl];
        int ip = s->part_idx_pre[i], jp = s->part_idx_pre[j];
        if (jp > ip) {
            int b = ip == 0 ? 0 : s->Nsum_pre[ip - 1];
            for (int o = b; o < s->Nsum_pre[ip]; o++)
                if (jp == s->Lpb_pre[o]) { dv[nl] = dv_old[o]; dt[nl] = dt_old[o]; dr[nl] = dr_old[o]; }
        } else if (jp < ip) {
            int b = jp == 0 ? 0 : s->Nsum_pre[jp - 1];
            for (int o = b; o < s->Nsum_pre[jp]; o++)
                if (ip == s->Lpb_pre[o]) {
                    dv[nl] = mul3(-1.0, dv_old[o]);
                    dt[nl] = mul3(-1.0, dt_old[o]);
                    dr[nl] = mul3(-1.0, dr_old[o]);
                }
        }
    }
}

/* Hierarchical history carry: the old owner of a pair is the old row that
 * holds it; search both old rows (the ownership rule mixes index and level). */
static void inherit_history_hgrid(nbo_scene* s, d3* dv, d3* dv_old, d3* dt, d3* dt_old, d3* dr,
                                  d3* dr_old) {
    for (int nl = 0; nl < s->npairs; nl++) {
        int i = s->Lpa[nl], j = s->Lpb[nl];
        int ip = s->part_idx_pre[i], jp = s->part_idx_pre[j];
        int b = ip == 0 ? 0 : s->Nsum_pre[ip - 1];
        int found = 0;
        for (int o = b; o < s->Nsum_pre[ip]; o++)
            if (jp == s->Lpb_pre[o]) { dv[nl] = dv_old[o]; dt[nl] = dt_old[o]; dr[nl] = dr_old[o]; found = 1; }
        if (found) continue;
        b = jp == 0 ? 0 : s->Nsum_pre[jp - 1];
        for (int o = b; o < s->Nsum_pre[jp]; o++)
            if (ip == s->Lpb_pre[o]) {
                dv[nl] = mul3(-1.0, dv_old[o]);
                dt[nl] = mul3(-1.0, dt_old[o]);
                dr[nl] = mul3(-1.0, dr_old[o]);
            }
    }
}

static void swap_i(int** a, int** b) { int* t = *a; *a = *b; *b = t; }
static void swap_d3(d3** a, d3** b) { d3* t = *a; *a = *b; *b = t; }

/* DEMGrid::CreateContList, src/dem_grid.cu:680-749.  The reference swaps
 * the history pointers it receives by value: the carried history lands in
 * the caller's Dv_pre and the caller's Dv is zeroed. */
static int create_list_all(nbo_scene* s) {
    int N = s->N, BL = s->BL;
    swap_i(&s->Lpb, &s->Lpb_pre);
    swap_i(&s->Nsum, &s->Nsum_pre);
    /* InitNList, src/dem_grid.cu:439-450 */
    memset(s->Ng, 0, N * sizeof(int));
    memset(s->Ni, 0, N * sizeof(int));
    size_t clear = s->hw;
    memset(s->Lpa, 0xFF, clear * sizeof(int));
    memset(s->Lpb, 0xFF, clear * sizeof(int));
    memset(s->Anei, 0xFF, (size_t)N * BL * sizeof(int));
    int ovf = s->levels > 1 ? create_anei_hgrid(s) : create_anei(s);
    if (ovf) return 1;
    int acc = 0;
    for (int i = 0; i < N; i++) { acc += s->Ng[i]; s->Nsum[i] = acc; }
    s->npairs = acc;
    if ((size_t)acc > s->hw) s->hw = (size_t)acc;
    create_cont_list(s);
    /* local swap: write into the caller's *_pre buffers */
    if (s->levels > 1)
        inherit_history_hgrid(s, s->Dv_pre, s->Dv, s->Dt_pre, s->Dt, s->Dr_pre, s->Dr);
    else
        inherit_history(s, s->Dv_pre, s->Dv, s->Dt_pre, s->Dt, s->Dr_pre, s->Dr);
    memset(s->Dv, 0, s->hw * sizeof(d3));
    memset(s->Dt, 0, s->hw * sizeof(d3));
    memset(s->Dr, 0, s->hw * sizeof(d3));
    return 0;
}

/* per-clump member lists in ascending sorted-index order: the order
 * thrust::sort_by_key + reduce_by_key visit them (src/dem_clumpsphere.cu:123-147) */
static void build_members(nbo_scene* s) {
    memset(s->mem_start, 0, (s->K + 1) * sizeof(int));
    for (int i = 0; i < s->N; i++) s->mem_start[s->clump_id[i] + 1]++;
    for (int k = 0; k < s->K; k++) s->mem_start[k + 1] += s->mem_start[k];
    int* cur = (int*)xcalloc(s->K, sizeof(int));
    for (int k = 0; k < s->K; k++) cur[k] = s->mem_start[k];
    for (int i = 0; i < s->N; i++) s->mem_order[cur[s->clump_id[i]]++] = i;
    free(cur);
}

/* the rebuild block of RunSimulationClump, src/dem_simulation_clump.cu:124-176 */
static int rebuild(nbo_scene* s) {
    if (s->levels > 1) cell_index_hgrid(s); else cell_index(s);
    sort_by_cell(s);
    find_beg_end(s);
    gather_d3(s, s->pos);
    gather_d3(s, s->local);
    gather_d(s, s->radius);
    gather_d(s, s->mass);
    gather_i(s, s->clump_id);
    if (s->levels > 1) gather_i(s, s->level);
    for (int f = 0; f < 6; f++)
        for (int h = 0; h < 3; h++) gather_d3(s, s->wc_hist[f][h]);
    for (int f = 0; f < 3; f++)
        for (int h = 0; h < 3; h++) gather_d3(s, s->cy_hist[f][h]);
    if (s->is_intruder) {
        gather_d3(s, s->pe_Dv);
        gather_d3(s, s->pe_Dt);
        gather_d3(s, s->pe_Dr);
    }
    int rc = create_list_all(s);
    if (rc) return rc;
    s->update = 0;
    memset(s->cum, 0, s->N * sizeof(d3));
    build_members(s);
    s->rebuilds++;
    return 0;
}

/* ---------------------------------------------------------------------------
 * contact laws
 * ------------------------------------------------------------------------- */

/* ContactForce_clump_cuk, src/dem_force_clump.cu:3-163 */
static void pair_force(nbo_scene* s) {
    double dt = s->dt;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
    for (int i = 0; i < s->npairs; i++) {
        int pI = s->Lpa[i], pJ = s->Lpb[i];
        if (pI < 0 || pJ < 0) continue;
        int cI = s->clump_id[pI], cJ = s->clump_id[pJ];
        if (cI == cJ) continue;
        d3 Dist = sub3(s->pos[pJ], s->pos[pI]);
        d3 H = s->Dv_pre[i], Mr = s->Dr_pre[i], Mt = s->Dt_pre[i];
        double DistS = Dist.x * Dist.x + Dist.y * Dist.y + Dist.z * Dist.z;
        double DistL = sqrt(DistS);
        double rI = s->radius[pI], rJ = s->radius[pJ];
        double Dn = rI + rJ - DistL;
        if (!(Dn > 0.0)) continue;
        double DistR = 1.0 / DistL;
        d3 DistU = mul3(DistR, Dist);
        double Ap = 0.50 * (rI * rI - rJ * rJ + DistS) * DistR;
        double An = DistL - Ap;
        double Rij = rI * rJ / (rI + rJ);
        double Mij = s->mass[pI] * s->mass[pJ] / (s->mass[pI] + s->mass[pJ]);
        double Kn = 2.0 * s->E * sqrt(Rij * Dn) / (3.0 * (1.0 - s->nu * s->nu));
        double Cn = s->damping * sqrt(Kn * Mij);
        double Ks = 2.0 * s->E / (1.0 + s->nu) / (2.0 - s->nu) * sqrt(Rij * Dn);
        double Cs = s->damping * sqrt(Ks * Mij);
        double br = s->beta * Rij;
        double Kr = 0.25 * Kn * br * br;
        double Cr = 0.25 * Cn * br * br;
        double Kt = 0.50 * Ks * br * br;
        double Ct = 0.50 * Cs * br * br;
        double mI[3][3], mJ[3][3];
        quat2ivdcm(s->cq[cI], mI);
        quat2ivdcm(s->cq[cJ], mJ);
        d3 ARMi = map3(mI, s->local[pI]);
        d3 ARMj = map3(mJ, s->local[pJ]);
        ARMi = add3(ARMi, mul3(Ap, DistU));
        ARMj = sub3(ARMj, mul3(An, DistU));
        d3 Vrel = sub3(s->cvel[cJ], s->cvel[cI]);
        d3 Vrot = sub3(cross3(s->cw[cJ], ARMj), cross3(s->cw[cI], ARMi));
        if (s->sphere & SPH_KIN)   /* ContactForce_cuk, src/dem_force_particle.cu:87-89 */
            Vrot = add3(mul3(An, cross3(DistU, s->cw[cJ])), mul3(Ap, cross3(DistU, s->cw[cI])));
        d3 Vtot = add3(Vrel, Vrot);
        double ERR = dot3(DistU, Vtot);
        d3 Vnor = mul3(ERR, DistU);
        d3 Vtan = sub3(Vtot, Vnor);
        d3 nf = add3(mul3(Kn * Dn, DistU), mul3(Cn, Vnor));
        double nfL = length3(nf);
        d3 Ds = mul3(dt, Vtan);
        d3 tf = add3(add3(mul3(-Ks, Ds), mul3(Cs, Vtan)), H);
        double tfL = length3(tf);
        d3 th;
        if (tfL > nfL * s->mu) {
            tf = mul3(s->mu * nfL * (1.0 / tfL), tf);
            th = tf;
        } else {
            th = sub3(tf, mul3(Cs, Vtan));
        }
        d3 coh = mul3(s->cohesion * br * br, DistU);
        s->CacheFc[i] = add3(sub3(mul3(-1.0, nf), tf), coh);
        d3 ct = cross3(DistU, tf);
        d3 tc = mul3(-Ap, ct);
        d3 tc2 = mul3(-An, ct);
        d3 Dth = mul3(dt, sub3(s->cw[cI], s->cw[cJ]));
        double DthL = dot3(Dth, DistU);
        d3 DthT = mul3(DthL, DistU);
        d3 DthR = sub3(Dth, DthT);
        d3 rm = add3(mul3(Kr, DthR), Mr), rh;
        double rmL = length3(rm);
        if (rmL > 0.525 * s->beta * Rij * nfL) {
            rm = mul3(0.525 * s->beta * Rij * nfL * (1.0 / rmL), rm);
            rh = rm;
        } else {
            rh = rm;
            rm = sub3(rm, mul3(Cr * (1.0 / dt), DthR));
        }
        d3 tm = add3(mul3(Kt, DthT), Mt), tw;
        double tmL = length3(tm);
        if (tmL > 0.65 * s->mu * s->beta * Rij * nfL) {
            tm = mul3(0.65 * s->mu * s->beta * Rij * nfL * (1.0 / tmL), tm);
            tw = tm;
        } else {
            tw = tm;
            tm = sub3(tm, mul3(Ct * (1.0 / dt), DthT));
        }
        s->CacheTc[i] = sub3(sub3(tc, rm), tm);
        s->CacheTc2[i] = add3(add3(tc2, rm), tm);
        s->Dv[i] = th;
        s->Dt[i] = tw;
        s->Dr[i] = rh;
        s->CacheFcn[i] = mul3(-1.0, nf);
        s->CacheCpt[i] = add3(s->pos[pI], mul3(Ap, DistU));
    }
}

/* SumContForce_clump, src/dem_force_clump.cu:165-191 */
static void sum_cont_force(nbo_scene* s) {
    int BL = s->BL;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->N; i++) {
        int* rr = row(s->Aref, BL, i);
        d3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
        for (int g = 0; g < s->Ng[i]; g++) {
            F = add3(F, s->CacheFc[rr[g]]);
            T = add3(T, s->CacheTc[rr[g]]);
        }
        for (int g = BL - s->Ni[i]; g < BL; g++) {
            F = sub3(F, s->CacheFc[rr[g]]);
            T = add3(T, s->CacheTc2[rr[g]]);
        }
        s->Fc[i] = F;
        s->Tc[i] = T;
    }
}

/* The shared wall law: ForceWall_Cube_clump_cuk (src/dem_force_cube_wall_clump.cu:
 * 16-183).  The cylinder wall uses the same law (ForceWall_cuk,
 * src/dem_force_cylind_wall.cu:3-139) with DistU = RVn/|RVn| and Ap = |RVn|. */
static void wall_law(nbo_scene* s, int i, d3 RVo, d3 DistU, double Ap, double Dn, d3 Wv, d3 Ww,
                     d3* Dv_pre, d3* Dt_pre, d3* Dr_pre, d3* Dv, d3* Dt, d3* Dr, int memless) {
    double dt = s->dt;
    int c = s->clump_id[i];
    d3 H = Dv_pre[i], Mr = Dr_pre[i], Mt = Dt_pre[i];
    if (memless) H = Mr = Mt = mk3(0, 0, 0);
    double Rij = s->radius[i], Mij = s->mass[i];
    double Kn = 2.0 * s->E * sqrt(Rij * Dn) / (3.0 * (1.0 - s->nu * s->nu));
    double Cn = s->damping * sqrt(Kn * Mij);
    double Ks = 2.0 * s->E / (1.0 + s->nu) / (2.0 - s->nu) * sqrt(Rij * Dn);
    double Cs = 2.0 * s->damping * sqrt(Ks * Mij);
    double br = s->beta * Rij;
    double Kr = 0.25 * Kn * br * br;
    double Cr = 0.25 * Cn * br * br;
    double Kt = 0.50 * Ks * br * br;
    double Ct = 0.50 * Cs * br * br;
    double m[3][3];
    quat2ivdcm(s->cq[c], m);
    d3 Arm = map3(m, s->local[i]);
    Arm = add3(mul3(-1.0, Arm), mul3(Ap, DistU));
    d3 Vwall = cross3(Ww, RVo);
    d3 Vrel = sub3(s->cvel[c], Wv);
    d3 Vrot = sub3(cross3(Arm, s->cw[c]), Vwall);
    if (s->sphere & SPH_KIN)   /* the sphere walls, src/dem_force_cylind_wall.cu:55, dem_force_cube_wall.cu:55 */
        Vrot = sub3(mul3(Ap, cross3(DistU, s->cw[c])), Vwall);
    d3 Vtot = add3(Vrel, Vrot);
    double ERR = dot3(DistU, Vtot);
    d3 Vnor = mul3(ERR, DistU);
    d3 Vtan = sub3(Vtot, Vnor);
    d3 nf = add3(mul3(Kn * Dn, DistU), mul3(Cn, Vnor));
    double nfL = length3(nf);
    d3 Ds = mul3(dt, Vtan);
    d3 tf = add3(add3(mul3(-Ks, Ds), mul3(Cs, Vtan)), H);
    double tfL = length3(tf);
    d3 th;
    if (tfL > nfL * s->mu) {
        tf = mul3(s->mu * nfL * (1.0 / tfL), tf);
        th = tf;
    } else {
        th = sub3(tf, mul3(Cs, Vtan));
    }
    s->Fw[i] = add3(add3(s->Fw[i], nf), tf);
    s->Tw[i] = sub3(s->Tw[i], mul3(Ap, cross3(DistU, tf)));
    /* the sphere cube wall stops here: its moment update and history
     * writes are commented out (src/dem_force_cube_wall.cu:137-141) */
    if (memless) return;
    d3 Dth = mul3(dt, sub3(s->cw[c], Ww));
    double DthL = dot3(Dth, DistU);
    d3 DthT = mul3(DthL, DistU);
    d3 DthR = sub3(Dth, DthT);
    d3 rm = add3(mul3(Kr, DthR), Mr), rh;
    double rmL = length3(rm);
    if (rmL > 0.525 * s->beta * Rij * nfL) {
        rm = mul3(0.525 * s->beta * Rij * nfL * (1.0 / rmL), rm);
        rh = rm;
    } else {
        rh = rm;
        rm = sub3(rm, mul3(Cr * (1.0 / dt), DthR));
    }
    d3 tm = add3(mul3(Kt, DthT), Mt), tw;
    double tmL = length3(tm);
    if (tmL > 0.65 * s->mu * s->beta * Rij * nfL) {
        tm = mul3(0.65 * s->mu * s->beta * Rij * nfL * (1.0 / tmL), tm);
        tw = tm;
    } else {
        tw = tm;
        tm = sub3(tm, mul3(Ct * (1.0 / dt), DthT));
    }
    s->Tw[i] = sub3(sub3(s->Tw[i], rm), tm);
    Dv[i] = th;
    Dt[i] = tw;
    Dr[i] = rh;
}

static int finite3(d3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

/* CubeWallInteraction_clump_cuk, src/dem_force_cube_wall_clump.cu:185-298 */
static int cube_wall(nbo_scene* s) {
    int bad = 0;
    d3 hl = s->cube_half;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(| : bad)
    for (int i = 0; i < s->N; i++) {
        int c = s->clump_id[i];
        if (c < 0 || c >= s->K) { bad = 1; continue; }
        d3 RV = sub3(s->pos[i], s->cube_c);
        double ex = RV.x, ey = RV.y, ez = RV.z, r = s->radius[i];
        d3 X = mk3(1, 0, 0), Y = mk3(0, 1, 0), Z = mk3(0, 0, 1);
        d3 RVbx = sub3(RV, mul3(ex, X)), RVtx = mul3(ex, X);
        d3 RVby = sub3(RV, mul3(ey, Y)), RVty = mul3(ey, Y);
        d3 RVbz = sub3(RV, mul3(ez, Z)), RVtz = mul3(ez, Z);
        struct { int on; d3 RVo, n; } f[6];
        f[0].on = ex > 0 && ex + r - hl.x > 0;
        f[0].RVo = add3(mul3(hl.x / fabs(ex), RVtx), RVbx); f[0].n = mk3(-1, 0, 0);
        f[1].on = ex < 0 && ex - r + hl.x < 0;
        f[1].RVo = f[0].RVo; f[1].n = mk3(1, 0, 0);
        f[2].on = ey > 0 && ey + r - hl.y > 0;
        f[2].RVo = add3(mul3(hl.y / fabs(ey), RVty), RVby); f[2].n = mk3(0, -1, 0);
        f[3].on = ey < 0 && ey - r + hl.y < 0;
        f[3].RVo = f[2].RVo; f[3].n = mk3(0, 1, 0);
        f[4].on = ez > 0 && ez + r - hl.z > 0;
        f[4].RVo = add3(mul3(hl.z / fabs(ez), RVtz), RVbz); f[4].n = mk3(0, 0, -1);
        f[5].on = ez < 0 && ez - r + hl.z < 0;
        f[5].RVo = f[4].RVo; f[5].n = mk3(0, 0, 1);
        /* face order of the reference: UpX, LowX, UpY, LowY, UpZ, LowZ */
        for (int k = 0; k < 6; k++) {
            if (!f[k].on) continue;
            d3 RVn = sub3(RV, f[k].RVo);
            double Ap = dot3(RVn, f[k].n);
            double Dn = r - Ap;
            d3 n = f[k].n;
            int memless = (s->sphere & SPH_CUBE) != 0;
            if (memless) {
                /* CubeWallInteraction_cuk / ForceWall_Cube_cuk
                 * (src/dem_force_cube_wall.cu:24-40,175-296): the normal and
                 * lever from RVn itself */
                Dn = r - length3(RVn);
                double DistL = sqrt(RVn.x * RVn.x + RVn.y * RVn.y + RVn.z * RVn.z);
                n = mul3(1.0 / DistL, RVn);
                Ap = DistL;
            }
            if (Dn <= 0.0) continue;
            wall_law(s, i, f[k].RVo, n, Ap, Dn, s->cube_v, s->cube_w,
                     s->wc_hist_pre[k][0], s->wc_hist_pre[k][1], s->wc_hist_pre[k][2],
                     s->wc_hist[k][0], s->wc_hist[k][1], s->wc_hist[k][2], memless);
        }
        if (!finite3(s->Fw[i]) || !finite3(s->Tw[i])) bad = 1;
    }
    return bad;
}

/* Closed cylinder wall with clump kinematics: the region tests of
 * CylindWallInteraction_cuk (src/dem_force_cylind_wall.cu:152-237) and the
 * wall law above. Regions: 0 bottom cap (ERR<0), 1 top cap, 2 side. */
static void cylinder_wall(nbo_scene* s) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->N; i++) {
        d3 ax = s->cyl_axis;
        d3 RV = sub3(s->pos[i], s->cyl_c);
        double ERR = dot3(RV, ax), r = s->radius[i];
        d3 RVb = sub3(RV, mul3(ERR, ax));
        d3 RVt = mul3(ERR, ax);
        double nrm = length3(RVb);
        double d_cap = fabs(ERR) - s->cyl_H + r;
        double d_side = nrm - s->cyl_R + r;
        for (int k = 0; k < 3; k++) {
            d3 RVo;
            if (k == 0) { if (!(d_cap >= 1e-14 && ERR < 0)) continue; RVo = add3(mul3(s->cyl_H / fabs(ERR), RVt), RVb); }
            else if (k == 1) { if (!(d_cap >= 1e-14 && ERR > 0)) continue; RVo = add3(mul3(s->cyl_H / fabs(ERR), RVt), RVb); }
            else { if (!(d_side >= 1e-14)) continue; RVo = add3(mul3(s->cyl_R / nrm, RVb), RVt); }
            d3 RVn = sub3(RV, RVo);
            double DistL0 = length3(RVn);
            double Dn = r - DistL0;
            if (!(Dn > 0.0)) continue;
            double DistL = sqrt(RVn.x * RVn.x + RVn.y * RVn.y + RVn.z * RVn.z);
            d3 DistU = mul3(1.0 / DistL, RVn);
            wall_law(s, i, RVo, DistU, DistL, Dn, s->cyl_v, s->cyl_w,
                     s->cy_hist_pre[k][0], s->cy_hist_pre[k][1], s->cy_hist_pre[k][2],
                     s->cy_hist[k][0], s->cy_hist[k][1], s->cy_hist[k][2], 0);
        }
    }
}

/* GetSphereIntruderContact, src/dem_sphere_intruder.cuh:20-51 */
typedef struct { d3 normal, surfaceArm, normalGapVector; double gap, overlap, particleArm; } sic;
static sic sphere_contact(d3 p, double r, d3 c, double R, d3 fallback) {
    sic o;
    d3 cv = sub3(p, c);
    double cd = length3(cv);
    if (cd > 1.0e-15) o.normal = mul3(1.0 / cd, cv);
    else {
        o.normal = norm3(fallback);
        if (length3(o.normal) < 1.0e-15) o.normal = mk3(0, 0, 1);
    }
    o.surfaceArm = mul3(R, o.normal);
    o.gap = cd - R;
    o.overlap = r - o.gap;
    o.particleArm = o.gap;
    o.normalGapVector = mul3(o.particleArm, o.normal);
    return o;
}

/* PrePenetrator, src/dem_contact_penetrator.cu:8-84 */
static void pre_penetrator(nbo_scene* s) {
    int touched = 0;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(| : touched)
    for (int i = 0; i < s->N; i++) {
        s->LcFlg[i] = 0;
        if (s->intr_shape == 1) {
            sic c = sphere_contact(s->pos[i], s->radius[i], s->intr_p, s->intr_R, s->intr_axis);
            if (c.overlap > 0.0) {
                s->RVo_i[i] = c.surfaceArm;
                s->RVn_i[i] = c.normalGapVector;
                s->LcFlg[i] = 1;
                if (s->intr_wait) touched = 1;
            }
            continue;
        }
        double LatDx = s->cell[0];
        d3 pv = s->intr_axis;
        d3 RV = sub3(s->pos[i], s->intr_p);
        double ERR = dot3(RV, pv);
        d3 RVn = mk3(0, 0, 0), RVo = mk3(0, 0, 0);
        int enter = 0;
        if (fabs(ERR) < (s->intr_H + 0.80 * LatDx)) {
            d3 RVb = sub3(RV, mul3(ERR, pv));
            double nrm = length3(RVb);
            if (nrm < (s->intr_R + 0.80 * LatDx)) {
                d3 RVt = mul3(ERR, pv);
                if (fabs(ERR) < s->intr_H) {
                    RVo = add3(mul3(1.0 / nrm * s->intr_R, RVb), RVt);
                } else if (nrm < s->intr_R) {
                    RVo = add3(mul3(1.0 / fabs(ERR) * s->intr_H, RVt), RVb);
                } else {
                    RVo = add3(mul3(1.0 / nrm * s->intr_R, RVb), mul3(1.0 / fabs(ERR) * s->intr_H, RVt));
                }
                RVn = sub3(RV, RVo);
                enter = 1;
            }
        }
        if (enter) {
            double DistL = sqrt(RVn.x * RVn.x + RVn.y * RVn.y + RVn.z * RVn.z);
            double Dn = s->radius[i] - DistL;
            if (Dn > 0.0) {
                s->RVo_i[i] = RVo;
                s->RVn_i[i] = RVn;
                s->LcFlg[i] = 1;
            }
        }
    }
    if (touched && s->intr_state == 0) s->intr_state = 1;
}

/* ForcePene_clump_cuk, src/dem_force_penetrator_clump.cu:4-182 */
static void pene_force(nbo_scene* s) {
    double dt = s->dt;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < s->N; i++) {
        if (s->LcFlg[i] == 0) continue;
        int c = s->clump_id[i];
        d3 Dist = s->RVn_i[i];
        d3 H = s->pe_Dv_pre[i], Mr = s->pe_Dr_pre[i], Mt = s->pe_Dt_pre[i];
        double DistS = Dist.x * Dist.x + Dist.y * Dist.y + Dist.z * Dist.z;
        double DistL = sqrt(DistS);
        double Dn = s->radius[i] - DistL;
        sic sc;
        if (s->intr_shape == 1) {
            sc = sphere_contact(s->pos[i], s->radius[i], s->intr_p, s->intr_R, s->intr_axis);
            Dist = sc.normalGapVector;
            DistL = sc.particleArm;
            Dn = sc.overlap;
        }
        if (!(Dn > 0.0)) continue;
        d3 DistU = s->intr_shape == 1 ? sc.normal : mul3(1.0 / DistL, Dist);
        double Ap = DistL;
        double Rij = s->radius[i];
        if (s->intr_shape == 1) Rij = s->radius[i] * s->intr_R / (s->radius[i] + s->intr_R);
        double Mij = s->mass[i];
        if (s->intr_motion == 1) Mij = s->mass[i] * s->intr_prop.w / (s->mass[i] + s->intr_prop.w);
        double Kn = 2.0 * s->E * sqrt(Rij * Dn) / (3.0 * (1.0 - s->nu * s->nu));
        double Cn = s->damping * sqrt(Kn * Mij);
        double Ks = 2.0 * s->E / (1.0 + s->nu) / (2.0 - s->nu) * sqrt(Rij * Dn);
        double Cs = s->damping * sqrt(Ks * Mij);
        double br = s->beta * Rij;
        double Kr = 0.25 * Kn * br * br;
        double Cr = 0.25 * Cn * br * br;
        double Kt = 0.50 * Ks * br * br;
        double Ct = 0.50 * Cs * br * br;
        double m[3][3];
        quat2ivdcm(s->cq[c], m);
        d3 Arm = map3(m, s->local[i]);
        Arm = add3(mul3(-1.0, Arm), mul3(Ap, DistU));
        d3 Vwall = cross3(s->intr_w, s->RVo_i[i]);
        d3 Vrel = sub3(s->cvel[c], s->intr_v);
        d3 Vrot = sub3(cross3(Arm, s->cw[c]), Vwall);
        if (s->sphere & SPH_KIN)   /* ForcePene_cuk, src/dem_force_penetrator.cu:83-84 */
            Vrot = sub3(mul3(Ap, cross3(DistU, s->cw[c])), Vwall);
        d3 Vtot = add3(Vrel, Vrot);
        double ERR = dot3(DistU, Vtot);
        d3 Vnor = mul3(ERR, DistU);
        d3 Vtan = sub3(Vtot, Vnor);
        d3 nf = add3(mul3(Kn * Dn, DistU), mul3(Cn, Vnor));
        double nfL = length3(nf);
        d3 Ds = mul3(dt, Vtan);
        d3 tf = add3(add3(mul3(-Ks, Ds), mul3(Cs, Vtan)), H);
        double tfL = length3(tf);
        d3 th;
        if (tfL > nfL * s->mu) {
            tf = mul3(s->mu * nfL * (1.0 / tfL), tf);
            th = tf;
        } else {
            th = sub3(tf, mul3(Cs, Vtan));
        }
        /* the clump law has no cohesion here; the sphere driver's adds
         * -Cohesion (beta R*)^2 n (src/dem_force_penetrator.cu:119-123) */
        d3 coh = (s->sphere & SPH_KIN) ? mul3(((-s->cohesion) * br) * br, DistU) : mk3(0, 0, 0);
        s->Fi[i] = (s->sphere & SPH_KIN) ? add3(add3(nf, tf), coh) : add3(nf, tf);
        s->Ti[i] = mul3(-Ap, cross3(DistU, tf));
        s->peneTc[i] = mul3(-1.0, cross3(s->RVo_i[i], add3(add3(nf, tf), coh)));
        s->Fcn_i[i] = nf;
        s->Fct_i[i] = tf;
        d3 Dth = mul3(dt, sub3(s->cw[c], s->intr_w));
        double DthL = dot3(Dth, DistU);
        d3 DthT = mul3(DthL, DistU);
        d3 DthR = sub3(Dth, DthT);
        d3 rm = add3(mul3(Kr, DthR), Mr), rh;
        double rmL = length3(rm);
        if (rmL > 0.525 * s->beta * Rij * nfL) {
            rm = mul3(0.525 * s->beta * Rij * nfL * (1.0 / rmL), rm);
            rh = rm;
        } else {
            rh = rm;
            rm = sub3(rm, mul3(Cr * (1.0 / dt), DthR));
        }
        d3 tm = add3(mul3(Kt, DthT), Mt), tw;
        double tmL = length3(tm);
        if (tmL > 0.65 * s->mu * s->beta * Rij * nfL) {
            tm = mul3(0.65 * s->mu * s->beta * Rij * nfL * (1.0 / tmL), tm);
            tw = tm;
        } else {
            tw = tm;
            tm = sub3(tm, mul3(Ct * (1.0 / dt), DthT));
        }
        s->Ti[i] = sub3(sub3(s->Ti[i], rm), tm);
        s->peneTc[i] = add3(add3(s->peneTc[i], rm), tm);
        s->pe_Dv[i] = th;
        s->pe_Dt[i] = tw;
        s->pe_Dr[i] = rh;
        s->Tcn_i[i] = cross3(nf, Arm);
        s->Tct_i[i] = sub3(sub3(cross3(tf, Arm), rm), tm);
    }
}

/* SumForce_cuk x2 (src/dem_force_penetrator.cu:189-248): the summation tree
 * of <<<128,128>>> followed by <<<1,1024>>>, reproduced exactly. */
static d3 block_tree(d3* v, int n) {
    /* shared-memory halving down to 32, then warp shuffle-down over lane 0..31 */
    for (int off = n >> 1; off >= 32; off >>= 1)
        for (int t = 0; t < off; t++) v[t] = add3(v[t], v[t + off]);
    d3 lane[32];
    for (int t = 0; t < 32; t++) lane[t] = v[t];
    for (int off = 16; off > 0; off >>= 1)
        for (int t = 0; t < 32; t++) {
            if (t + off < 32) lane[t] = add3(lane[t], lane[t + off]);
        }
    return lane[0];
}
static d3 sum_force(const d3* F, int N) {
    d3 cache[128];
    d3 sm[128];
    for (int b = 0; b < 128; b++) {
        for (int t = 0; t < 128; t++) {
            d3 f = mk3(0, 0, 0);
            for (int n = b * 128 + t; n < N; n += 128 * 128) f = add3(f, F[n]);
            sm[t] = f;
        }
        cache[b] = block_tree(sm, 128);
    }
    d3* big = (d3*)xcalloc(1024, sizeof(d3));
    for (int t = 0; t < 128; t++) big[t] = cache[t];
    d3 r = block_tree(big, 1024);
    free(big);
    return r;
}

/* IntegratePene_Before_cuk, src/dem_integrate_penetrator.cu:3-50 */
static void pene_integrate_before(nbo_scene* s) {
    double Dt = s->dt;
    if (s->intr_motion == 1 && (!s->intr_wait || s->intr_state != 0)) {
        d3 F = mul3(-1.0 / s->intr_prop.w, s->totFc);
        F.z = F.z + s->gravity;
        s->intr_p = add3(add3(s->intr_p, mul3(Dt, s->intr_v)), mul3(0.5 * Dt * Dt, F));
        s->intr_v = add3(s->intr_v, mul3(0.5 * Dt, F));
    } else {
        s->intr_p = add3(s->intr_p, mul3(Dt, s->intr_v));
    }
}

/* Integrate_After_cuk, src/dem_integrate_penetrator.cu:86-113 */
static void pene_integrate_after(nbo_scene* s) {
    if (s->intr_wait && s->intr_state == 1) s->intr_state = 2;
    d3 reaction = mul3(-1.0, s->totFc);
    if (s->intr_motion == 1 && (!s->intr_wait || s->intr_state != 0)) {
        d3 F = mul3(1.0 / s->intr_prop.w, reaction);
        F.z = F.z + s->gravity;
        s->intr_v = add3(s->intr_v, mul3(0.5 * s->dt, F));
    }
    s->reaction = reaction;
    s->reaction_t = s->totTc;
}

/* ComputeTorqueFromWorldPos_Kernel + reduce_by_key,
 * src/dem_clumpsphere.cu:86-151 */
static void sum_force_on_clump(nbo_scene* s) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int k = 0; k < s->K; k++) {
        int b = s->mem_start[k], e = s->mem_start[k + 1];
        if (b == e) continue;
        d3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
        for (int m = b; m < e; m++) {
            int i = s->mem_order[m];
            d3 r = sub3(s->pos[i], s->cpos[k]);
            d3 fs = s->totF[i], ts = s->totT[i];
            d3 tcn;
            tcn.x = ts.x + (r.y * fs.z - r.z * fs.y);
            tcn.y = ts.y + (r.z * fs.x - r.x * fs.z);
            tcn.z = ts.z + (r.x * fs.y - r.y * fs.x);
            F = (m == b) ? fs : add3(F, fs);
            T = (m == b) ? tcn : add3(T, tcn);
        }
        s->cFc[k] = F;
        s->cTc[k] = T;
    }
}

/* ---------------------------------------------------------------------------
 * the step, src/dem_simulation_clump.cu:110-225
 * ------------------------------------------------------------------------- */
static void exchange_walls(nbo_scene* s) {
    /* DEMWallCube::ForceExchange, src/dem_cube_wall.cu:157-206 */
    for (int f = 0; f < 6; f++)
        for (int h = 0; h < 3; h++) {
            swap_d3(&s->wc_hist[f][h], &s->wc_hist_pre[f][h]);
            memset(s->wc_hist[f][h], 0, s->N * sizeof(d3));
        }
    for (int f = 0; f < 3; f++)
        for (int h = 0; h < 3; h++) {
            swap_d3(&s->cy_hist[f][h], &s->cy_hist_pre[f][h]);
            memset(s->cy_hist[f][h], 0, s->N * sizeof(d3));
        }
}

int nbo_step(nbo_scene* s, int nsteps) {
    for (int it = 0; it < nsteps; it++) {
        if (s->sphere) {
            sphere_integrate_before(s);
        } else {
            clump_integrate_before(s);
            update_pos(s);
        }
        if (s->is_intruder) pene_integrate_before(s);
        int rebuilt = s->update != 0 || s->step == s->start_step;
        if (rebuilt) {
            int rc = rebuild(s);
            if (rc) return rc;
            if (s->sphere) memset(s->scum, 0, s->K * sizeof(d3));
        }
        /* the cylinder and split drivers exchange the pair histories on
         * every step, after a rebuild too (src/dem_simulation_cylind.cu:141):
         * the carried histories are cleared */
        if (!rebuilt || (s->sphere & SPH_RESET)) {
            /* DEMForce::ForceExchange, src/dem_force.cu:88-98 */
            swap_d3(&s->Dv, &s->Dv_pre);
            swap_d3(&s->Dt, &s->Dt_pre);
            swap_d3(&s->Dr, &s->Dr_pre);
            memset(s->Dv, 0, s->hw * sizeof(d3));
            memset(s->Dt, 0, s->hw * sizeof(d3));
            memset(s->Dr, 0, s->hw * sizeof(d3));
        }
        exchange_walls(s);
        if (s->is_intruder) {
            swap_d3(&s->pe_Dv, &s->pe_Dv_pre);
            swap_d3(&s->pe_Dt, &s->pe_Dt_pre);
            swap_d3(&s->pe_Dr, &s->pe_Dr_pre);
            memset(s->pe_Dv, 0, s->N * sizeof(d3));
            memset(s->pe_Dt, 0, s->N * sizeof(d3));
            memset(s->pe_Dr, 0, s->N * sizeof(d3));
        }
        /* ForceZero: DEMForce (src/dem_force.cu:75-86) and the walls */
        memset(s->CacheFc, 0, s->hw * sizeof(d3));
        memset(s->CacheTc, 0, s->hw * sizeof(d3));
        memset(s->CacheTc2, 0, s->hw * sizeof(d3));
        memset(s->CacheFcn, 0, s->hw * sizeof(d3));
        memset(s->CacheCpt, 0, s->hw * sizeof(d3));
        memset(s->Fw, 0, s->N * sizeof(d3));
        memset(s->Tw, 0, s->N * sizeof(d3));
        pair_force(s);
        sum_cont_force(s);
        if (s->is_wall) {
            if (s->has_cube && cube_wall(s)) return 2;
            if (s->has_cyl) cylinder_wall(s);
        }
        memset(s->Fi, 0, s->N * sizeof(d3));
        memset(s->Ti, 0, s->N * sizeof(d3));
        memset(s->peneTc, 0, s->N * sizeof(d3));
        if (s->is_intruder) {
            memset(s->Fcn_i, 0, s->N * sizeof(d3));
            memset(s->Fct_i, 0, s->N * sizeof(d3));
            memset(s->Tcn_i, 0, s->N * sizeof(d3));
            memset(s->Tct_i, 0, s->N * sizeof(d3));
            pre_penetrator(s);
            pene_force(s);
            s->totFc = sum_force(s->Fi, s->N);
            s->totTc = sum_force(s->peneTc, s->N);
            pene_integrate_after(s);
        }
        /* SumAllForces_cuk, src/dem_clump.cu:89-101 */
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int i = 0; i < s->N; i++) {
            s->totF[i] = add3(add3(s->Fc[i], s->Fw[i]), s->Fi[i]);
            s->totT[i] = add3(add3(s->Tc[i], s->Tw[i]), s->Ti[i]);
        }
        sum_force_on_clump(s);
        if (s->sphere) sphere_integrate_after(s);
        else clump_integrate_after(s);
        s->step++;
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * getters
 * ------------------------------------------------------------------------- */
int nbo_num_pairs(const nbo_scene* s) { return s->npairs; }
int nbo_step_count(const nbo_scene* s) { return s->step; }
int nbo_rebuild_count(const nbo_scene* s) { return s->rebuilds; }

static void put3(double* dst, const d3* src, int n) {
    for (int i = 0; i < n; i++) { dst[3 * i] = src[i].x; dst[3 * i + 1] = src[i].y; dst[3 * i + 2] = src[i].z; }
}

void nbo_get_sub(const nbo_scene* s, int* part_fix, int* clump_id, double* pos, double* radius) {
    if (part_fix) memcpy(part_fix, s->part_fix, s->N * sizeof(int));
    if (clump_id) memcpy(clump_id, s->clump_id, s->N * sizeof(int));
    if (pos) put3(pos, s->pos, s->N);
    if (radius) memcpy(radius, s->radius, s->N * sizeof(double));
}

void nbo_get_clumps(const nbo_scene* s, double* pos, double* vel, double* quat, double* angvel,
                    double* force, double* torque) {
    if (pos) put3(pos, s->cpos, s->K);
    if (vel) put3(vel, s->cvel, s->K);
    if (angvel) put3(angvel, s->cw, s->K);
    if (force) put3(force, s->cFc, s->K);
    if (torque) put3(torque, s->cTc, s->K);
    if (quat)
        for (int k = 0; k < s->K; k++) {
            quat[4 * k] = s->cq[k].x; quat[4 * k + 1] = s->cq[k].y;
            quat[4 * k + 2] = s->cq[k].z; quat[4 * k + 3] = s->cq[k].w;
        }
}

void nbo_get_sub_forces(const nbo_scene* s, double* fc, double* tc, double* fw, double* tw,
                        double* fi, double* ti) {
    if (fc) put3(fc, s->Fc, s->N);
    if (tc) put3(tc, s->Tc, s->N);
    if (fw) put3(fw, s->Fw, s->N);
    if (tw) put3(tw, s->Tw, s->N);
    if (fi) put3(fi, s->Fi, s->N);
    if (ti) put3(ti, s->Ti, s->N);
}

void nbo_get_pairs(const nbo_scene* s, int* lpa, int* lpb) {
    if (lpa) memcpy(lpa, s->Lpa, s->npairs * sizeof(int));
    if (lpb) memcpy(lpb, s->Lpb, s->npairs * sizeof(int));
}

void nbo_get_rows(const nbo_scene* s, int* anei, int* ng, int* ni) {
    if (anei) memcpy(anei, s->Anei, (size_t)s->N * s->BL * sizeof(int));
    if (ng) memcpy(ng, s->Ng, s->N * sizeof(int));
    if (ni) memcpy(ni, s->Ni, s->N * sizeof(int));
}

void nbo_get_pair_caches(const nbo_scene* s, double* cfc, double* cfcn, double* cpt, double* dv,
                         double* dt, double* dr) {
    if (cfc) put3(cfc, s->CacheFc, s->npairs);
    if (cfcn) put3(cfcn, s->CacheFcn, s->npairs);
    if (cpt) put3(cpt, s->CacheCpt, s->npairs);
    if (dv) put3(dv, s->Dv, s->npairs);
    if (dt) put3(dt, s->Dt, s->npairs);
    if (dr) put3(dr, s->Dr, s->npairs);
}

/* CalFcnChain_cuk, src/dem_force_particle.cu:238-268 (rows zeroed first) */
void nbo_get_chain(const nbo_scene* s, double* fcn_rows, double* cpt_rows) {
    int BL = s->BL;
    memset(fcn_rows, 0, (size_t)s->N * BL * 3 * sizeof(double));
    memset(cpt_rows, 0, (size_t)s->N * BL * 3 * sizeof(double));
    for (int i = 0; i < s->N; i++) {
        const int* rr = s->Aref + (size_t)i * BL;
        double* fr = fcn_rows + (size_t)i * BL * 3;
        double* cr = cpt_rows + (size_t)i * BL * 3;
        for (int g = 0; g < s->Ng[i]; g++) {
            d3 f = s->CacheFcn[rr[g]], c = s->CacheCpt[rr[g]];
            fr[3 * g] = f.x; fr[3 * g + 1] = f.y; fr[3 * g + 2] = f.z;
            cr[3 * g] = c.x; cr[3 * g + 1] = c.y; cr[3 * g + 2] = c.z;
        }
        for (int g = BL - s->Ni[i]; g < BL; g++) {
            d3 f = mul3(-1.0, s->CacheFcn[rr[g]]), c = s->CacheCpt[rr[g]];
            fr[3 * g] = f.x; fr[3 * g + 1] = f.y; fr[3 * g + 2] = f.z;
            cr[3 * g] = c.x; cr[3 * g + 1] = c.y; cr[3 * g + 2] = c.z;
        }
    }
}

void nbo_get_intruder(const nbo_scene* s, double* pos, double* vel, double* totf, double* tott,
                      double* reaction, int* state) {
    if (pos) put3(pos, &s->intr_p, 1);
    if (vel) put3(vel, &s->intr_v, 1);
    if (totf) put3(totf, &s->totFc, 1);
    if (tott) put3(tott, &s->totTc, 1);
    if (reaction) put3(reaction, &s->reaction, 1);
    if (state) *state = s->intr_state;
}

void nbo_get_intruder_diag(const nbo_scene* s, double* fcn, double* fct, double* tcn, double* tct) {
    if (fcn) put3(fcn, s->Fcn_i, s->N);
    if (fct) put3(fct, s->Fct_i, s->N);
    if (tcn) put3(tcn, s->Tcn_i, s->N);
    if (tct) put3(tct, s->Tct_i, s->N);
}
