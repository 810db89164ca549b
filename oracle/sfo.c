/*
 * sfo.c -- CPU oracle (FP64, single thread) for the SoftFlow hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA implementation.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Citations are to the reference project (ramc77/SoftFlow) by path:line.
 * Expression order follows the reference so that the results agree bit for
 * bit with the reference engine when both are compiled with -O2
 * -ffp-contract=off (no -ffast-math).
 */
#include "sfo.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define Q 9
static const double W[Q] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                            1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
static const int CX[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int CY[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int OPP[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const double PI_ = 3.14159265358979323846;

enum { CT_FLUID = 0, CT_SOLID = 1, CT_INLET = 2, CT_OUTLET = 3 };
enum { BT_INLET_OUTLET = 0, BT_PERIODIC = 1, BT_CLOSED = 2 };

typedef struct { double x, y; } v2;
static inline v2 vadd(v2 a, v2 b) { v2 r = {a.x + b.x, a.y + b.y}; return r; }
static inline v2 vsub(v2 a, v2 b) { v2 r = {a.x - b.x, a.y - b.y}; return r; }
static inline v2 vmul(v2 a, double s) { v2 r = {a.x * s, a.y * s}; return r; }
static inline v2 vdiv(v2 a, double s) { v2 r = {a.x / s, a.y / s}; return r; }
static inline double vdot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline double vcross(v2 a, v2 b) { return a.x * b.y - a.y * b.x; }
static inline double vnorm(v2 a) { return sqrt(a.x * a.x + a.y * a.y); }

typedef struct {
    int off, n, type;
    sf_membrane m;
    double rest_area, rest_perimeter;
    double wlc_kBT_p, wlc_k_pow;
    int has_prev;
    int periodic_nx;
} capsule_t;

/* circle (a, b) radius c, or rectangle [a, c] x [b, d] */
typedef struct { int rect; double a, b, c, d; } obstacle_t;
typedef struct { int x, y, q; double qf; } ibb_link_t;

struct sfo_sim {
    sf_params p;
    int nobs;
    obstacle_t obs[64];
    int nlinks;
    ibb_link_t* links;
    int chem_on;
    sf_chemistry chem;
    double *released, *absorbed, *Mp, *gamma;
    int nx, ny, N;
    double *f, *ftmp, *rho, *ux, *uy, *Fx, *Fy;
    int* flags;
    /* markers (capsule-major, node-minor) */
    int ncaps, cap_caps, M, cap_M;
    capsule_t* caps;
    v2 *pos, *vel, *frc;
    double *rest_len, *rest_ang, *rest_ds, *prev_len;
    int* offsets;
    /* scalar */
    double *g, *gtmp, *C;
    int last_capped;
    /* contact bookkeeping */
    int *pair_count, *pair_list, pair_len, pair_cap;
    double phi_tbl[1025];
};

/* ------------------------------------------------------------------ */
/* Parameters                                                         */
/* ------------------------------------------------------------------ */

/* Defaults of reference src/core/parameters.h:41-342 for the fields used. */
void sf_params_default(sf_params* p) {
    memset(p, 0, sizeof(*p));
    p->nx = 200; p->ny = 50;
    p->collision = SF_BGK;
    p->tau = 0.8; p->rho0 = 1.0;
    p->mrt_se = 1.4; p->mrt_s_eps = 1.4; p->mrt_sq = 1.4;
    p->max_lattice_force = 0.01;
    p->ibm_iterations = 1;
    p->dt = 1.0;
    p->rep_epsilon = 0.05; p->rep_sigma = 1.0; p->rep_r_cut = 3.5; p->rep_power = 4;
    p->scalar_D = 0.01;
    p->boundary_type = BT_PERIODIC;
    p->inlet_velocity = 0.02;
    p->outlet_density = 1.0;
    p->top_wall_velocity = 0.0;
    p->bottom_wall_velocity = 0.0;
    p->use_interpolated_bb = 0;
}

/* Defaults of reference MembraneParams (parameters.h:82-136). */
void sf_membrane_default(sf_membrane* m) {
    memset(m, 0, sizeof(*m));
    m->model = SF_HOOKEAN;
    m->k_stretch = 0.1; m->G_s = 0.1; m->C_skalak = 1.0;
    m->wlc_L_max_ratio = 2.2;
    m->k_bend = 0.005;
    m->k_area = 0.5; m->k_perimeter = 0.1; m->gamma_visc = 0.01; m->eta_membrane = 0.05;
}

/* ------------------------------------------------------------------ */
/* Peskin 4-point delta with the 1024-bin table                        */
/* reference src/coupling/delta_function.h:18-59                       */
/* ------------------------------------------------------------------ */

static double phi_exact(double r) {
    double ar = fabs(r);
    if (ar <= 1.0) return 0.125 * (3.0 - 2.0 * ar + sqrt(1.0 + 4.0 * ar - 4.0 * ar * ar));
    if (ar <= 2.0) return 0.125 * (5.0 - 2.0 * ar - sqrt(-7.0 + 12.0 * ar - 4.0 * ar * ar));
    return 0.0;
}

static double phi_tab(const double* tbl, double r) {
    double ar = fabs(r);
    if (ar >= 2.0) return 0.0;
    double idx = ar * (1024 * 0.5);
    int i = (int)idx;
    if (i >= 1024) return 0.0;
    double frac = idx - (double)i;
    return tbl[i] * (1.0 - frac) + tbl[i + 1] * frac;
}

static double g_phi_tbl[1025];
static int g_phi_init = 0;
double sfo_phi(double r) {
    if (!g_phi_init) {
        for (int i = 0; i <= 1024; ++i) g_phi_tbl[i] = phi_exact(2.0 * (double)i / 1024);
        g_phi_init = 1;
    }
    return phi_tab(g_phi_tbl, r);
}

/* ------------------------------------------------------------------ */
/* Lattice                                                             */
/* ------------------------------------------------------------------ */

static inline double feq(int q, double rho, double ux, double uy) {
    /* reference src/lbm/lattice.h:35-39 */
    const double cs2 = 1.0 / 3.0;
    const double cs4 = cs2 * cs2;
    double eu = (double)CX[q] * ux + (double)CY[q] * uy;
    double uu = ux * ux + uy * uy;
    return W[q] * rho * (1.0 + eu / cs2 + (eu * eu) / (2.0 * cs4) - uu / (2.0 * cs2));
}

sfo_sim* sfo_create(const sf_params* p) {
    sfo_sim* s = (sfo_sim*)calloc(1, sizeof(sfo_sim));
    s->p = *p;
    s->nx = p->nx; s->ny = p->ny; s->N = p->nx * p->ny;
    size_t N = (size_t)s->N;
    s->f = (double*)calloc(N * Q, sizeof(double));
    s->ftmp = (double*)calloc(N * Q, sizeof(double));
    s->rho = (double*)calloc(N, sizeof(double));
    s->ux = (double*)calloc(N, sizeof(double));
    s->uy = (double*)calloc(N, sizeof(double));
    s->Fx = (double*)calloc(N, sizeof(double));
    s->Fy = (double*)calloc(N, sizeof(double));
    s->flags = (int*)calloc(N, sizeof(int));
    s->g = (double*)calloc(N * Q, sizeof(double));
    s->gtmp = (double*)calloc(N * Q, sizeof(double));
    s->C = (double*)calloc(N, sizeof(double));
    s->offsets = (int*)calloc(1, sizeof(int));
    for (int i = 0; i <= 1024; ++i) s->phi_tbl[i] = phi_exact(2.0 * (double)i / 1024);
    return s;
}

void sfo_destroy(sfo_sim* s) {
    if (!s) return;
    free(s->f); free(s->ftmp); free(s->rho); free(s->ux); free(s->uy);
    free(s->Fx); free(s->Fy); free(s->flags); free(s->g); free(s->gtmp); free(s->C);
    free(s->caps); free(s->pos); free(s->vel); free(s->frc);
    free(s->rest_len); free(s->rest_ang); free(s->rest_ds); free(s->prev_len);
    free(s->offsets); free(s->pair_count); free(s->pair_list); free(s->links);
    free(s->released); free(s->absorbed); free(s->Mp); free(s->gamma);
    free(s);
}

/* reference lattice_field.cpp:28-73 */
void sfo_compute_macroscopic(sfo_sim* s) {
    const int N = s->N;
    for (int n = 0; n < N; ++n) {
        if (s->flags[n] == CT_SOLID) {
            s->rho[n] = 0.0; s->ux[n] = 0.0; s->uy[n] = 0.0;
            continue;
        }
        double r = 0.0, vx = 0.0, vy = 0.0;
        for (int q = 0; q < Q; ++q) {
            double fi = s->f[q * N + n];
            r += fi;
            vx += fi * (double)CX[q];
            vy += fi * (double)CY[q];
        }
        s->rho[n] = r;
        if (r > 1e-15) {
            s->ux[n] = (vx + 0.5 * s->Fx[n]) / r;
            s->uy[n] = (vy + 0.5 * s->Fy[n]) / r;
        } else {
            s->ux[n] = 0.0; s->uy[n] = 0.0;
        }
    }
}

/* reference bgk_collision.cpp:15-86 */
static void collide_bgk(sfo_sim* s) {
    const int N = s->N;
    const double om = 1.0 / s->p.tau;
    const double om1 = 1.0 - om;
    const double guo = 1.0 - 0.5 * om;
    const double inv_cs2 = 3.0, inv_cs4 = 9.0;
    for (int n = 0; n < N; ++n) {
        if (s->flags[n] != CT_FLUID) continue;
        const double r = s->rho[n], vx = s->ux[n], vy = s->uy[n];
        const double fx = s->Fx[n], fy = s->Fy[n];
        const double uu = vx * vx + vy * vy;
        const double uu_term = -0.5 * inv_cs2 * uu;
        for (int q = 0; q < Q; ++q) {
            const double eqx = (double)CX[q], eqy = (double)CY[q];
            const double eu = eqx * vx + eqy * vy;
            double f_eq = W[q] * r * (1.0 + eu * inv_cs2 + 0.5 * eu * eu * inv_cs4 + uu_term);
            double term_x = (eqx - vx) * inv_cs2 + (eu * inv_cs4) * eqx;
            double term_y = (eqy - vy) * inv_cs2 + (eu * inv_cs4) * eqy;
            double F_i = guo * W[q] * (term_x * fx + term_y * fy);
            s->f[q * N + n] = om1 * s->f[q * N + n] + om * f_eq + F_i;
        }
    }
}

/* reference regularized_bgk.cpp:15-93 */
static void collide_regularized(sfo_sim* s) {
    const int N = s->N;
    const double omega = 1.0 / s->p.tau;
    const double cs2 = 1.0 / 3.0;
    const double cs4_2 = 2.0 * cs2 * cs2;
    for (int n = 0; n < N; ++n) {
        if (s->flags[n] != CT_FLUID) continue;
        double rho = s->rho[n], ux = s->ux[n], uy = s->uy[n];
        double Fx = s->Fx[n], Fy = s->Fy[n];
        double fe[Q], fl[Q];
        for (int q = 0; q < Q; ++q) {
            fe[q] = feq(q, rho, ux, uy);
            fl[q] = s->f[q * N + n];
        }
        double jx = 0.0, jy = 0.0, pxx = 0.0, pxy = 0.0, pyy = 0.0;
        for (int q = 0; q < Q; ++q) {
            double fneq = fl[q] - fe[q];
            jx += fneq * CX[q];
            jy += fneq * CY[q];
            pxx += fneq * CX[q] * CX[q];
            pxy += fneq * CX[q] * CY[q];
            pyy += fneq * CY[q] * CY[q];
        }
        for (int q = 0; q < Q; ++q) {
            double Qxx = CX[q] * CX[q] - cs2;
            double Qxy = CX[q] * CY[q];
            double Qyy = CY[q] * CY[q] - cs2;
            double fneq_reg = W[q] * ((CX[q] * jx + CY[q] * jy) / cs2 +
                                      (Qxx * pxx + 2.0 * Qxy * pxy + Qyy * pyy) / cs4_2);
            double eu = CX[q] * ux + CY[q] * uy;
            double Fi = (1.0 - 0.5 * omega) * W[q] *
                        ((CX[q] - ux + eu * CX[q] / cs2) * Fx / cs2 +
                         (CY[q] - uy + eu * CY[q] / cs2) * Fy / cs2);
            s->f[q * N + n] = fe[q] + (1.0 - omega) * fneq_reg + Fi;
        }
    }
}

/* reference mrt_collision.cpp:31-140 (Lallemand-Luo basis, Guo source in
 * moment space). */
static void collide_mrt(sfo_sim* s) {
    const int N = s->N;
    const double sn = 1.0 / s->p.tau;
    const double s1 = s->p.mrt_se, s2 = s->p.mrt_s_eps, s4 = s->p.mrt_sq, s6 = s->p.mrt_sq;
    for (int n = 0; n < N; ++n) {
        if (s->flags[n] != CT_FLUID) continue;
        const double r = s->rho[n], vx = s->ux[n], vy = s->uy[n];
        const double fx = s->Fx[n], fy = s->Fy[n];
        double* f = s->f;
        double f0 = f[0 * N + n], f1 = f[1 * N + n], f2 = f[2 * N + n];
        double f3 = f[3 * N + n], f4 = f[4 * N + n], f5 = f[5 * N + n];
        double f6 = f[6 * N + n], f7 = f[7 * N + n], f8 = f[8 * N + n];
        double m0 = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
        double m1 = -4 * f0 - f1 - f2 - f3 - f4 + 2 * f5 + 2 * f6 + 2 * f7 + 2 * f8;
        double m2 = 4 * f0 - 2 * f1 - 2 * f2 - 2 * f3 - 2 * f4 + f5 + f6 + f7 + f8;
        double m3 = f1 - f3 + f5 - f6 - f7 + f8;
        double m4 = -2 * f1 + 2 * f3 + f5 - f6 - f7 + f8;
        double m5 = f2 - f4 + f5 + f6 - f7 - f8;
        double m6 = -2 * f2 + 2 * f4 + f5 + f6 - f7 - f8;
        double m7 = f1 - f2 + f3 - f4;
        double m8 = f5 - f6 + f7 - f8;
        double uu = vx * vx + vy * vy;
        double meq1 = -2.0 * r + 3.0 * r * uu;
        double meq2 = r - 3.0 * r * uu;
        double meq4 = -r * vx;
        double meq6 = -r * vy;
        double meq7 = r * (vx * vx - vy * vy);
        double meq8 = r * vx * vy;
        double uF = vx * fx + vy * fy;
        double Sb1 = 6.0 * uF, Sb2 = -6.0 * uF;
        double Sb3 = fx, Sb4 = -fx, Sb5 = fy, Sb6 = -fy;
        double Sb7 = 2.0 * (vx * fx - vy * fy);
        double Sb8 = vx * fy + vy * fx;
        m1 = m1 - s1 * (m1 - meq1) + (1.0 - s1 * 0.5) * Sb1;
        m2 = m2 - s2 * (m2 - meq2) + (1.0 - s2 * 0.5) * Sb2;
        m3 = m3 + Sb3;
        m4 = m4 - s4 * (m4 - meq4) + (1.0 - s4 * 0.5) * Sb4;
        m5 = m5 + Sb5;
        m6 = m6 - s6 * (m6 - meq6) + (1.0 - s6 * 0.5) * Sb6;
        m7 = m7 - sn * (m7 - meq7) + (1.0 - sn * 0.5) * Sb7;
        m8 = m8 - sn * (m8 - meq8) + (1.0 - sn * 0.5) * Sb8;
        f0 = m0 / 9.0 - m1 / 9.0 + m2 / 9.0;
        f1 = m0 / 9.0 - m1 / 36.0 - m2 / 18.0 + m3 / 6.0 - m4 / 6.0 + m7 / 4.0;
        f2 = m0 / 9.0 - m1 / 36.0 - m2 / 18.0 + m5 / 6.0 - m6 / 6.0 - m7 / 4.0;
        f3 = m0 / 9.0 - m1 / 36.0 - m2 / 18.0 - m3 / 6.0 + m4 / 6.0 + m7 / 4.0;
        f4 = m0 / 9.0 - m1 / 36.0 - m2 / 18.0 - m5 / 6.0 + m6 / 6.0 - m7 / 4.0;
        f5 = m0 / 9.0 + m1 / 18.0 + m2 / 36.0 + m3 / 6.0 + m4 / 12.0 + m5 / 6.0 + m6 / 12.0 + m8 / 4.0;
        f6 = m0 / 9.0 + m1 / 18.0 + m2 / 36.0 - m3 / 6.0 - m4 / 12.0 + m5 / 6.0 + m6 / 12.0 - m8 / 4.0;
        f7 = m0 / 9.0 + m1 / 18.0 + m2 / 36.0 - m3 / 6.0 - m4 / 12.0 - m5 / 6.0 - m6 / 12.0 + m8 / 4.0;
        f8 = m0 / 9.0 + m1 / 18.0 + m2 / 36.0 + m3 / 6.0 + m4 / 12.0 - m5 / 6.0 - m6 / 12.0 - m8 / 4.0;
        f[0 * N + n] = f0; f[1 * N + n] = f1; f[2 * N + n] = f2;
        f[3 * N + n] = f3; f[4 * N + n] = f4; f[5 * N + n] = f5;
        f[6 * N + n] = f6; f[7 * N + n] = f7; f[8 * N + n] = f8;
    }
}

/* Pull streaming with periodic folding (reference lbm_solver.cpp:72-104,
 * 212-235): out-of-range sources fall back to the node itself. */
static void stream(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    const int px = s->p.boundary_type == BT_PERIODIC, py = s->p.periodic_y;
    for (int q = 0; q < Q; ++q) {
        for (int y = 0; y < ny; ++y) {
            for (int x = 0; x < nx; ++x) {
                int n = y * nx + x;
                int xs = x - CX[q], ys = y - CY[q];
                if (px) xs = (xs + nx) % nx;
                if (py) ys = (ys + ny) % ny;
                int oob = (!px && (xs < 0 || xs >= nx)) || (!py && (ys < 0 || ys >= ny));
                int src = oob ? n : ys * nx + xs;
                s->ftmp[q * N + n] = s->f[q * N + src];
            }
        }
    }
    double* t = s->f; s->f = s->ftmp; s->ftmp = t;
}

/* Halfway bounce-back over the SOLID nodes (reference bounce_back.cpp:12-41). */
static void bounce_back(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    for (int n = 0; n < N; ++n) {
        if (s->flags[n] != CT_SOLID) continue;
        int x = n % nx, y = n / nx;
        for (int q = 1; q < Q; ++q) {
            int xn = x - CX[q], yn = y - CY[q];
            if (s->p.boundary_type == BT_PERIODIC) xn = (xn + nx) % nx;
            if (s->p.periodic_y) yn = (yn + ny) % ny;
            if (xn < 0 || xn >= nx || yn < 0 || yn >= ny) continue;
            if (s->flags[yn * nx + xn] == CT_SOLID) continue;
            s->f[OPP[q] * N + yn * nx + xn] = s->f[q * N + n];
        }
    }
}

/* Moving top / bottom walls after the halfway bounce-back (reference
 * moving_wall.cpp:14-64): the reflected population of each link into a wall
 * row loses 2 w_q rho_n (e_q . u_wall) / cs^2, rho_n of the fluid node from
 * the last macroscopic update. */
static void moving_wall_row(sfo_sim* s, int yw, double vel) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    const double cs2 = 1.0 / 3.0;
    for (int x = 0; x < nx; ++x) {
        if (s->flags[yw * nx + x] != CT_SOLID) continue;
        for (int q = 1; q < Q; ++q) {
            int xn = x - CX[q], yn = yw - CY[q];
            if (s->p.boundary_type == BT_PERIODIC) xn = (xn + nx) % nx;
            if (xn < 0 || xn >= nx || yn < 0 || yn >= ny) continue;
            if (s->flags[yn * nx + xn] == CT_SOLID) continue;
            double rho = s->rho[yn * nx + xn];
            double eu_wall = CX[q] * vel;
            s->f[OPP[q] * N + yn * nx + xn] = s->f[q * N + yw * nx + x]
                - 2.0 * W[q] * rho * eu_wall / cs2;
        }
    }
}

static void moving_walls(sfo_sim* s) {
    if (fabs(s->p.bottom_wall_velocity) > 1e-15) moving_wall_row(s, 0, s->p.bottom_wall_velocity);
    if (fabs(s->p.top_wall_velocity) > 1e-15) moving_wall_row(s, s->ny - 1, s->p.top_wall_velocity);
}

/* Obstacle::contains of CircleObstacle / RectObstacle
 * (geometry/circle_obstacle.h:11-15, rect_obstacle.h:9-16). */
static int obstacle_contains(const obstacle_t* o, double x, double y) {
    if (o->rect) return x >= o->a && x <= o->c && y >= o->b && y <= o->d;
    double dx = x - o->a, dy = y - o->b;
    return (dx * dx + dy * dy) <= o->c * o->c;
}

static double obstacle_sd(const obstacle_t* o, double x, double y);

void sfo_add_circle_pillar(sfo_sim* s, double cx, double cy, double radius) {
    obstacle_t o = {0, cx, cy, radius, 0.0};
    if (s->nobs < 64) s->obs[s->nobs++] = o;
}

void sfo_add_rect_pillar(sfo_sim* s, double x0, double y0, double x1, double y1) {
    obstacle_t o = {1, x0 < x1 ? x0 : x1, y0 < y1 ? y0 : y1, x0 > x1 ? x0 : x1, y0 > y1 ? y0 : y1};
    if (s->nobs < 64) s->obs[s->nobs++] = o;
}

/* InterpolatedBounceBack::initialize (interpolated_bounce_back.cpp:7-54):
 * every link of a non-SOLID node into a SOLID node, with the wall distance
 * found by bisection against the obstacles (1 where none is crossed). */
static void ibb_build(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny;
    s->nlinks = 0;
    int cap = 64;
    s->links = (ibb_link_t*)realloc(s->links, sizeof(ibb_link_t) * cap);
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) {
            if (s->flags[y * nx + x] == CT_SOLID) continue;
            for (int q = 1; q < Q; ++q) {
                int xn = x + CX[q], yn = y + CY[q];
                if (xn < 0 || xn >= nx || yn < 0 || yn >= ny) continue;
                if (s->flags[yn * nx + xn] != CT_SOLID) continue;
                double x0 = (double)x, y0 = (double)y, dx = (double)CX[q], dy = (double)CY[q];
                double min_q = 1.0;
                for (int k = 0; k < s->nobs; ++k) {
                    double lo = 0.0, hi = 1.0;
                    for (int it = 0; it < 20; ++it) {
                        double mid = 0.5 * (lo + hi);
                        double xm = x0 + mid * dx, ym = y0 + mid * dy;
                        if (obstacle_contains(&s->obs[k], xm, ym)) hi = mid;
                        else lo = mid;
                    }
                    if (hi < min_q) min_q = hi;
                }
                if (s->nlinks == cap) {
                    cap *= 2;
                    s->links = (ibb_link_t*)realloc(s->links, sizeof(ibb_link_t) * cap);
                }
                ibb_link_t l = {x, y, q, min_q};
                s->links[s->nlinks++] = l;
            }
        }
    }
}

/* InterpolatedBounceBack::apply (interpolated_bounce_back.cpp:56-96), links
 * in their build order. */
static void ibb_apply(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    const int pnx = s->p.boundary_type == BT_PERIODIC ? nx : 0;
    for (int i = 0; i < s->nlinks; ++i) {
        const ibb_link_t* l = &s->links[i];
        int x = l->x, y = l->y, q = l->q, opp = OPP[q];
        double qf = l->qf;
        if (qf < 0.5) {
            int xu = x - CX[q], yu = y - CY[q];
            if (pnx > 0) xu = ((xu % pnx) + pnx) % pnx;
            if (xu >= 0 && xu < nx && yu >= 0 && yu < ny) {
                s->f[opp * N + y * nx + x] = 2.0 * qf * s->f[q * N + y * nx + x]
                    + (1.0 - 2.0 * qf) * s->f[q * N + yu * nx + xu];
            } else {
                s->f[opp * N + y * nx + x] = s->f[q * N + y * nx + x];
            }
        } else {
            double inv2q = 1.0 / (2.0 * qf);
            s->f[opp * N + y * nx + x] = inv2q * s->f[q * N + y * nx + x]
                + (1.0 - inv2q) * s->f[opp * N + y * nx + x];
        }
    }
}

/* Zou-He velocity inlet (parabolic profile) on the INLET column and
 * pressure outlet on the OUTLET column, in the order of the reference's
 * node lists (zou_he_boundary.cpp:17-85: inlet nodes, then outlet nodes,
 * each by increasing y). */
static void zou_he(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
#define F(x, y, q) s->f[(q) * N + (y) * nx + (x)]
    for (int y = 0; y < ny; ++y) {
        const int x = 0;
        if (s->flags[y * nx + x] != CT_INLET) continue;
        double y_center = (double)ny * 0.5;
        double H = (double)(ny - 2);
        double y_norm = ((double)y - y_center) / (H * 0.5);
        double ux = s->p.inlet_velocity * (1.0 - y_norm * y_norm);
        double uy = 0.0;
        double f0 = F(x, y, 0), f2 = F(x, y, 2), f3 = F(x, y, 3);
        double f4 = F(x, y, 4), f6 = F(x, y, 6), f7 = F(x, y, 7);
        double rho = (f0 + f2 + f4 + 2.0 * (f3 + f6 + f7)) / (1.0 - ux);
        F(x, y, 1) = f3 + (2.0 / 3.0) * rho * ux;
        F(x, y, 5) = f7 + 0.5 * (f4 - f2) + (1.0 / 6.0) * rho * ux + 0.5 * rho * uy;
        F(x, y, 8) = f6 - 0.5 * (f4 - f2) + (1.0 / 6.0) * rho * ux - 0.5 * rho * uy;
    }
    for (int y = 0; y < ny; ++y) {
        const int x = nx - 1;
        if (s->flags[y * nx + x] != CT_OUTLET) continue;
        double rho = s->p.outlet_density;
        double f0 = F(x, y, 0), f1 = F(x, y, 1), f2 = F(x, y, 2);
        double f4 = F(x, y, 4), f5 = F(x, y, 5), f8 = F(x, y, 8);
        double ux = -1.0 + (f0 + f2 + f4 + 2.0 * (f1 + f5 + f8)) / rho;
        double uy = 0.0;
        F(x, y, 3) = f1 - (2.0 / 3.0) * rho * ux;
        F(x, y, 7) = f5 - 0.5 * (f4 - f2) - (1.0 / 6.0) * rho * ux - 0.5 * rho * uy;
        F(x, y, 6) = f8 + 0.5 * (f4 - f2) - (1.0 / 6.0) * rho * ux + 0.5 * rho * uy;
    }
#undef F
}

/* reference lbm_solver.cpp:172-207 (collide -> stream -> BB -> moving wall
 * -> Zou-He -> macroscopic) */
static void lbm_step(sfo_sim* s) {
    if (s->p.collision == SF_REGULARIZED) collide_regularized(s);
    else if (s->p.collision == SF_MRT) collide_mrt(s);
    else collide_bgk(s);
    stream(s);
    bounce_back(s);
    moving_walls(s);
    if (s->nlinks > 0) ibb_apply(s);
    if (s->p.boundary_type == BT_INLET_OUTLET) zou_he(s);
    sfo_compute_macroscopic(s);
}

/* ------------------------------------------------------------------ */
/* Advection-diffusion (reference advection_diffusion.cpp:84-223)      */
/* ------------------------------------------------------------------ */

static void adr_step(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    const double tau_s = 3.0 * s->p.scalar_D + 0.5;
    const double omega_s = 1.0 / tau_s;
    const double inv_cs2 = 1.0 / (1.0 / 3.0);
    /* collide (advection_diffusion.cpp:111-153) */
    for (int n = 0; n < N; ++n) {
        const double* src = s->g + (size_t)n * Q;
        double* dst = s->gtmp + (size_t)n * Q;
        if (s->flags[n] == CT_SOLID) {
            for (int q = 0; q < Q; ++q) dst[q] = src[q];
            continue;
        }
        const double C = s->C[n];
        const double ux = s->ux[n], uy = s->uy[n];
        for (int q = 0; q < Q; ++q) {
            const double eu = (double)CX[q] * ux + (double)CY[q] * uy;
            const double geq = W[q] * C * (1.0 + eu * inv_cs2);
            dst[q] = src[q] - omega_s * (src[q] - geq);
        }
    }
    /* stream with halfway BB (advection_diffusion.cpp:168-210) */
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) {
            const int n = y * nx + x;
            if (s->flags[n] == CT_SOLID) continue;
            for (int q = 0; q < Q; ++q) {
                int xs = x - CX[q], ys = y - CY[q];
                xs = ((xs % nx) + nx) % nx;
                if (s->p.scalar_periodic_y) ys = ((ys % ny) + ny) % ny;
                if (ys < 0 || ys >= ny) {
                    s->g[(size_t)n * Q + q] = s->gtmp[(size_t)n * Q + OPP[q]];
                    continue;
                }
                const int up = ys * nx + xs;
                if (s->flags[up] == CT_SOLID)
                    s->g[(size_t)n * Q + q] = s->gtmp[(size_t)n * Q + OPP[q]];
                else
                    s->g[(size_t)n * Q + q] = s->gtmp[(size_t)up * Q + q];
            }
        }
    }
    /* concentration (advection_diffusion.cpp:212-223) */
    for (int n = 0; n < N; ++n) {
        double C = 0.0;
        for (int q = 0; q < Q; ++q) C += s->g[(size_t)n * Q + q];
        s->C[n] = C;
    }
}

/* ------------------------------------------------------------------ */
/* Capsule chemistry (reference advection_diffusion.cpp:225-437)        */
/* ------------------------------------------------------------------ */

void sfo_set_chemistry(sfo_sim* s, const sf_chemistry* c) {
    s->chem = *c;
    s->chem_on = 1;
}

void sfo_chemistry_state(const sfo_sim* s, double* released, double* absorbed, double* Mp,
                         double* gamma) {
    for (int c = 0; c < s->ncaps; ++c) {
        if (released) released[c] = s->released ? s->released[c] : 0.0;
        if (absorbed) absorbed[c] = s->absorbed ? s->absorbed[c] : 0.0;
        if (Mp) Mp[c] = s->Mp ? s->Mp[c] : -1.0;
    }
    if (gamma)
        for (int k = 0; k < s->M; ++k) gamma[k] = s->gamma ? s->gamma[k] : 0.0;
}

static inline double chem_get(const double* v, int n, int type, double dflt) {
    return type < n ? v[type] : dflt;
}

/* per-capsule arrays as the first call sizes them (:231-234, :300-316) */
static void chem_init(sfo_sim* s) {
    if (s->released) return;
    s->released = (double*)calloc(s->ncaps > 0 ? s->ncaps : 1, sizeof(double));
    s->absorbed = (double*)calloc(s->ncaps > 0 ? s->ncaps : 1, sizeof(double));
    s->Mp = (double*)calloc(s->ncaps > 0 ? s->ncaps : 1, sizeof(double));
    s->gamma = (double*)calloc(s->M > 0 ? s->M : 1, sizeof(double));
    for (int c = 0; c < s->ncaps; ++c) {
        int type = s->caps[c].type;
        s->Mp[c] = -1.0;
        if (type < s->chem.n_M_p && s->chem.M_p_initial[type] > 0.0)
            s->Mp[c] = s->chem.M_p_initial[type];
    }
}

/* constant rates at the nearest node (:225-271) */
static void chem_source_sink(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny;
    for (int c = 0; c < s->ncaps; ++c) {
        const capsule_t* cp = &s->caps[c];
        int type = cp->type;
        double release = chem_get(s->chem.release, s->chem.n_release, type, 0.0);
        double absorb = chem_get(s->chem.absorb, s->chem.n_absorb, type, 0.0);
        for (int ni = 0; ni < cp->n; ++ni) {
            v2 pos = s->pos[cp->off + ni];
            int ix = (int)(pos.x + 0.5);
            int iy = (int)(pos.y + 0.5);
            ix = ix < 0 ? 0 : (ix > nx - 1 ? nx - 1 : ix);
            iy = iy < 0 ? 0 : (iy > ny - 1 ? ny - 1 : iy);
            int n = iy * nx + ix;
            s->C[n] += release;
            s->released[c] += release;
            double actual = (s->C[n] < absorb) ? s->C[n] : absorb;   /* std::min */
            s->C[n] -= actual;
            s->absorbed[c] += actual;
            for (int q = 0; q < Q; ++q) s->g[(size_t)n * Q + q] = W[q] * s->C[n];
        }
    }
}

/* leaching, Langmuir adsorption, Peskin-weighted exchange (:273-437) */
static void chem_physics(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, Lx = nx;
    for (int c = 0; c < s->ncaps; ++c) {
        const capsule_t* cp = &s->caps[c];
        int type = cp->type, Nn = cp->n;
        double k_L = chem_get(s->chem.k_leach, s->chem.n_k_leach, type, 0.0);
        double Ceq = chem_get(s->chem.C_eq, s->chem.n_C_eq, type, 0.0);
        double k_a = chem_get(s->chem.k_adsorb, s->chem.n_k_adsorb, type, 0.0);
        double k_d = chem_get(s->chem.k_desorb, s->chem.n_k_desorb, type, 0.0);
        double Gmax = chem_get(s->chem.Gamma_max, s->chem.n_Gamma_max, type, 1.0);
        double const_release = chem_get(s->chem.release, s->chem.n_release, type, 0.0);
        double const_absorb = chem_get(s->chem.absorb, s->chem.n_absorb, type, 0.0);
        for (int k = 0; k < Nn; ++k) {
            v2 pos = s->pos[cp->off + k];
            int kp = (k + 1) % Nn, km = (k - 1 + Nn) % Nn;
            v2 pp = s->pos[cp->off + kp], pm = s->pos[cp->off + km];
            double dxp = pp.x - pos.x, dyp = pp.y - pos.y;
            double dxm = pos.x - pm.x, dym = pos.y - pm.y;
            double ds = 0.5 * (sqrt(dxp * dxp + dyp * dyp) + sqrt(dxm * dxm + dym * dym));
            if (ds < 1e-12) ds = 1.0;
            int ix0 = (int)floor(pos.x), iy0 = (int)floor(pos.y);
            double C_surf = 0.0;
            for (int dy = -1; dy <= 2; ++dy) {
                int jy = iy0 + dy;
                if (jy < 0 || jy >= ny) continue;
                for (int dx = -1; dx <= 2; ++dx) {
                    int jx = ix0 + dx;
                    jx = ((jx % Lx) + Lx) % Lx;
                    double rx = pos.x - (double)(ix0 + dx);
                    double ry = pos.y - (double)jy;
                    double w = phi_tab(s->phi_tbl, rx) * phi_tab(s->phi_tbl, ry);
                    C_surf += s->C[jy * nx + jx] * w;
                }
            }
            double dC_leach = 0.0;
            if (k_L > 0.0) {
                dC_leach = k_L * (Ceq - C_surf);
                if (s->Mp[c] >= 0.0) {
                    if (dC_leach > 0.0) {
                        double available_per_ds = s->Mp[c] / ds;
                        dC_leach = (available_per_ds < dC_leach) ? available_per_ds : dC_leach;
                        s->Mp[c] -= dC_leach * ds;
                        if (s->Mp[c] < 0.0) s->Mp[c] = 0.0;
                    }
                }
            } else {
                double absorb_now = (C_surf < const_absorb) ? C_surf : const_absorb;
                dC_leach = const_release - absorb_now;
            }
            double dC_adsorb = 0.0;
            if (k_a > 0.0 || k_d > 0.0) {
                double* G = &s->gamma[cp->off + k];
                double dGamma = k_a * C_surf * (1.0 - *G / Gmax) - k_d * *G;
                double t = *G + dGamma;
                t = (t < Gmax) ? t : Gmax;              /* std::min(Gmax, t) */
                *G = (0.0 < t) ? t : 0.0;               /* std::max(0.0, t) */
                dC_adsorb = -dGamma;
            }
            double total_flux = dC_leach + dC_adsorb;
            if (total_flux == 0.0) continue;
            for (int dy = -1; dy <= 2; ++dy) {
                int jy = iy0 + dy;
                if (jy < 0 || jy >= ny) continue;
                for (int dx = -1; dx <= 2; ++dx) {
                    int jx = ix0 + dx;
                    jx = ((jx % Lx) + Lx) % Lx;
                    double rx = pos.x - (double)(ix0 + dx);
                    double ry = pos.y - (double)jy;
                    double w = phi_tab(s->phi_tbl, rx) * phi_tab(s->phi_tbl, ry);
                    if (w < 1e-15) continue;
                    int n = jy * nx + jx;
                    s->C[n] += total_flux * w * ds;
                    if (s->C[n] < 0.0) s->C[n] = 0.0;
                    for (int q = 0; q < Q; ++q) s->g[(size_t)n * Q + q] = W[q] * s->C[n];
                }
            }
            if (total_flux > 0.0) s->released[c] += total_flux * ds;
            else s->absorbed[c] -= total_flux * ds;
        }
    }
}

/* simulation.cpp:640-653 */
static void chemistry(sfo_sim* s) {
    if (!s->chem_on) return;
    int has_physics = s->chem.n_k_leach > 0 || s->chem.n_k_adsorb > 0;
    if (has_physics) {
        chem_init(s);
        chem_physics(s);
    } else if (s->chem.n_release > 0 || s->chem.n_absorb > 0) {
        chem_init(s);
        chem_source_sink(s);
    }
}

void sfo_set_concentration(sfo_sim* s, const double* C) {
    for (int n = 0; n < s->N; ++n) {
        s->C[n] = C[n];
        for (int q = 0; q < Q; ++q) s->g[(size_t)n * Q + q] = W[q] * C[n];
    }
}

/* ------------------------------------------------------------------ */
/* Capsules                                                            */
/* ------------------------------------------------------------------ */

static inline v2 min_image(const capsule_t* c, v2 a, v2 b) {
    /* reference capsule.h:129-137 */
    v2 d = vsub(a, b);
    if (c->periodic_nx > 0) {
        double Lx = (double)c->periodic_nx;
        if (d.x > 0.5 * Lx) d.x -= Lx;
        if (d.x < -0.5 * Lx) d.x += Lx;
    }
    return d;
}

#define NODE(c, i) s->pos[(c)->off + (i)]
static inline int nx_(const capsule_t* c, int i) { return (i + 1) % c->n; }
static inline int pv_(const capsule_t* c, int i) { return (i - 1 + c->n) % c->n; }

/* reference capsule.cpp:175-195 */
static double cap_area(const sfo_sim* s, const capsule_t* c) {
    const int n = c->n;
    if (c->periodic_nx > 0 && n > 0) {
        v2* uw = (v2*)malloc(sizeof(v2) * n);
        uw[0] = NODE(c, 0);
        for (int i = 1; i < n; ++i) uw[i] = vadd(uw[i - 1], min_image(c, NODE(c, i), NODE(c, i - 1)));
        double A = 0.0;
        for (int i = 0; i < n; ++i) A += vcross(uw[i], uw[(i + 1) % n]);
        free(uw);
        return 0.5 * fabs(A);
    }
    double A = 0.0;
    for (int i = 0; i < n; ++i) A += vcross(NODE(c, i), NODE(c, nx_(c, i)));
    return 0.5 * fabs(A);
}

/* reference capsule.cpp:197-204 */
static double cap_perimeter(const sfo_sim* s, const capsule_t* c) {
    double P = 0.0;
    for (int i = 0; i < c->n; ++i) P += vnorm(min_image(c, NODE(c, nx_(c, i)), NODE(c, i)));
    return P;
}

/* reference capsule.cpp:159-173 */
static v2 cap_centroid(const sfo_sim* s, const capsule_t* c) {
    if (c->periodic_nx > 0 && c->n > 0) {
        v2 ref = NODE(c, 0), sum = ref;
        for (int i = 1; i < c->n; ++i) sum = vadd(sum, vadd(ref, min_image(c, NODE(c, i), ref)));
        return vdiv(sum, (double)c->n);
    }
    v2 cc = {0.0, 0.0};
    for (int i = 0; i < c->n; ++i) cc = vadd(cc, NODE(c, i));
    return vdiv(cc, (double)c->n);
}

/* reference capsule.cpp:209-247: central second moments of area of the
 * polygon on nodes unwrapped across the periodic x boundary */
static void cap_moments(const sfo_sim* s, const capsule_t* c, double* mxx, double* myy,
                        double* mxy) {
    const int n = c->n;
    v2* p = (v2*)malloc(sizeof(v2) * (n > 0 ? n : 1));
    p[0] = NODE(c, 0);
    for (int i = 1; i < n; ++i) p[i] = vadd(p[i - 1], min_image(c, NODE(c, i), NODE(c, i - 1)));
    double A = 0.0, cx = 0.0, cy = 0.0;
    for (int i = 0; i < n; ++i) {
        v2 a = p[i], b = p[(i + 1) % n];
        double cr = a.x * b.y - b.x * a.y;
        A += cr;
        cx += (a.x + b.x) * cr;
        cy += (a.y + b.y) * cr;
    }
    A *= 0.5;
    *mxx = *myy = *mxy = 0.0;
    if (fabs(A) < 1e-15) { free(p); return; }
    cx /= (6.0 * A);
    cy /= (6.0 * A);
    for (int i = 0; i < n; ++i) {
        double x0 = p[i].x - cx, y0 = p[i].y - cy;
        v2 q = p[(i + 1) % n];
        double x1 = q.x - cx, y1 = q.y - cy;
        double cr = x0 * y1 - x1 * y0;
        *mxx += (x0 * x0 + x0 * x1 + x1 * x1) * cr;
        *myy += (y0 * y0 + y0 * y1 + y1 * y1) * cr;
        *mxy += (x0 * y1 + 2.0 * x0 * y0 + 2.0 * x1 * y1 + x1 * y0) * cr;
    }
    double sgn = (A > 0.0) ? 1.0 : -1.0;
    *mxx *= sgn / 12.0;
    *myy *= sgn / 12.0;
    *mxy *= sgn / 24.0;
    free(p);
}

/* reference capsule.cpp:249-258 (Taylor deformation of the equivalent ellipse) */
static double cap_deformation(const sfo_sim* s, const capsule_t* c) {
    if (c->n < 3) return 0.0;
    double mxx, myy, mxy;
    cap_moments(s, c, &mxx, &myy, &mxy);
    double tr = 0.5 * (mxx + myy);
    double dd = sqrt(0.25 * (mxx - myy) * (mxx - myy) + mxy * mxy);
    double J1 = tr + dd, t2 = tr - dd;
    double J2 = (t2 < 0.0) ? 0.0 : t2;
    double s1 = sqrt(J1), s2 = sqrt(J2);
    return (s1 + s2 > 1e-15) ? (s1 - s2) / (s1 + s2) : 0.0;
}

/* reference capsule.cpp:260-266 */
static double cap_inclination(const sfo_sim* s, const capsule_t* c) {
    if (c->n < 3) return 0.0;
    double mxx, myy, mxy;
    cap_moments(s, c, &mxx, &myy, &mxy);
    return 0.5 * atan2(2.0 * mxy, mxx - myy);
}

static void grow_markers(sfo_sim* s, int need) {
    if (need <= s->cap_M) return;
    int cap = s->cap_M ? s->cap_M : 64;
    while (cap < need) cap *= 2;
    s->pos = (v2*)realloc(s->pos, sizeof(v2) * cap);
    s->vel = (v2*)realloc(s->vel, sizeof(v2) * cap);
    s->frc = (v2*)realloc(s->frc, sizeof(v2) * cap);
    s->rest_len = (double*)realloc(s->rest_len, sizeof(double) * cap);
    s->rest_ang = (double*)realloc(s->rest_ang, sizeof(double) * cap);
    s->rest_ds = (double*)realloc(s->rest_ds, sizeof(double) * cap);
    s->prev_len = (double*)realloc(s->prev_len, sizeof(double) * cap);
    s->cap_M = cap;
}

/* Capsule constructor for the circle shape (reference capsule.cpp:7-141).
 * The capsule is built with periodic_nx = 0 and switched to periodic right
 * after construction (capsule_system.cpp:5-9), so the rest geometry uses
 * plain differences. */
int sfo_add_capsule(sfo_sim* s, double cx, double cy, double radius, int nn,
                    const sf_membrane* m, int type) {
    if (nn <= 0) {
        int n = (int)ceil(2.0 * PI_ * radius / 0.75);   /* capsule.h:14-17 */
        nn = n > 12 ? n : 12;
    }
    if (s->ncaps == s->cap_caps) {
        s->cap_caps = s->cap_caps ? 2 * s->cap_caps : 16;
        s->caps = (capsule_t*)realloc(s->caps, sizeof(capsule_t) * s->cap_caps);
    }
    grow_markers(s, s->M + nn);
    capsule_t* c = &s->caps[s->ncaps];
    memset(c, 0, sizeof(*c));
    c->off = s->M; c->n = nn; c->type = type; c->m = *m;
    c->periodic_nx = 0;
    for (int i = 0; i < nn; ++i) {
        double th = 2.0 * PI_ * i / nn;
        v2 r = {radius * cos(th), radius * sin(th)};
        v2 p = {cx + r.x, cy + r.y};
        NODE(c, i) = p;
        s->vel[c->off + i].x = 0.0; s->vel[c->off + i].y = 0.0;
        s->frc[c->off + i].x = 0.0; s->frc[c->off + i].y = 0.0;
    }
    for (int i = 0; i < nn; ++i) s->rest_len[c->off + i] = vnorm(vsub(NODE(c, nx_(c, i)), NODE(c, i)));
    for (int i = 0; i < nn; ++i) s->prev_len[c->off + i] = s->rest_len[c->off + i];
    c->has_prev = 0;
    c->rest_area = cap_area(s, c);
    c->rest_perimeter = cap_perimeter(s, c);
    c->wlc_kBT_p = m->wlc_kBT_p;
    c->wlc_k_pow = m->wlc_k_pow;
    if (m->model == SF_WLC && nn > 0) {
        double L0 = s->rest_len[c->off];
        double L_max = m->wlc_L_max_ratio * L0;
        double x0 = L0 / L_max;
        if (c->wlc_kBT_p <= 0.0) {
            double denom = 1.0 / (2.0 * (1.0 - x0) * (1.0 - x0) * (1.0 - x0)) + 1.0;
            c->wlc_kBT_p = m->G_s * L_max / (L0 * denom);
        }
        if (c->wlc_k_pow <= 0.0) {
            double F_wlc_rest = c->wlc_kBT_p * (1.0 / (4.0 * (1.0 - x0) * (1.0 - x0)) - 0.25 + x0);
            c->wlc_k_pow = F_wlc_rest * L0;
        }
    }
    for (int i = 0; i < nn; ++i) { s->rest_ang[c->off + i] = 0.0; s->rest_ds[c->off + i] = 0.0; }
    if (m->use_helfrich) {
        for (int i = 0; i < nn; ++i) {
            v2 e_prev = min_image(c, NODE(c, i), NODE(c, pv_(c, i)));
            v2 e_next = min_image(c, NODE(c, nx_(c, i)), NODE(c, i));
            s->rest_ds[c->off + i] = 0.5 * (vnorm(e_prev) + vnorm(e_next));
            s->rest_ang[c->off + i] = (m->kappa_0 != 0.0)
                ? m->kappa_0 * s->rest_ds[c->off + i]
                : atan2(vcross(e_prev, e_next), vdot(e_prev, e_next));
        }
    }
    /* periodic channel: capsules switch to minimum-image after construction */
    c->periodic_nx = s->nx;
    s->M += nn;
    s->ncaps += 1;
    s->offsets = (int*)realloc(s->offsets, sizeof(int) * (s->ncaps + 1));
    for (int k = 0; k <= s->ncaps; ++k) s->offsets[k] = (k < s->ncaps) ? s->caps[k].off : s->M;
    return s->ncaps - 1;
}

/* --- std::mt19937 + std::uniform_real_distribution<double>, restated ---
 * MT19937 (Matsumoto & Nishimura 1998) and the C++ generate_canonical
 * contract for a 32-bit engine and 53 mantissa bits: two draws combined as
 * (g1 + g2 * 2^32) / 2^64, clamped below 1, then a + (b - a) * u. */
typedef struct { uint32_t mt[624]; int idx; } mt19937_t;
static void mt_seed(mt19937_t* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}
static uint32_t mt_next(mt19937_t* g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}
static double mt_uniform(mt19937_t* g, double a, double b) {
    const double r = 4294967296.0;
    double sum = (double)mt_next(g);
    sum += (double)mt_next(g) * r;
    double u = sum / (r * r);
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    return u * (b - a) + a;
}

/* reference simulation.cpp:220-274 */
int sfo_add_capsule_random(sfo_sim* s, int count, double x0, double y0, double x1,
                           double y1, double rmin, double rmax, int nn,
                           const sf_membrane* m, int type, int seed, double min_gap,
                           int max_attempts, int check_walls) {
    mt19937_t g;
    mt_seed(&g, (uint32_t)seed);
    int placed = 0, attempts = 0;
    int total_max = max_attempts > 0 ? max_attempts : count * 500;
    while (placed < count && attempts < total_max) {
        double cx = mt_uniform(&g, x0, x1);
        double cy = mt_uniform(&g, y0, y1);
        double r = mt_uniform(&g, rmin, rmax);
        int overlap = 0;
        for (int c = 0; c < s->ncaps; ++c) {
            v2 oc = cap_centroid(s, &s->caps[c]);
            double orad = sqrt(s->caps[c].rest_area / PI_);
            v2 d = {cx - oc.x, cy - oc.y};
            if (vnorm(d) < r + orad + min_gap) { overlap = 1; break; }
        }
        if (check_walls) {
            if (cy - r < 0.0 + min_gap || cy + r > (double)(s->ny - 1) - min_gap) overlap = 1;
            for (int o = 0; o < s->nobs; ++o)                 /* simulation.cpp:256-261 */
                if (obstacle_sd(&s->obs[o], cx, cy) < r + min_gap) { overlap = 1; break; }
        }
        if (!overlap) {
            sfo_add_capsule(s, cx, cy, r, nn, m, type);
            placed++;
        }
        attempts++;
    }
    return placed;
}

/* reference capsule.cpp:149-157 and the per-law routines :320-671 */
static void membrane_forces(sfo_sim* s, capsule_t* c) {
    const int n = c->n;
    v2* F = s->frc + c->off;
    const v2* V = s->vel + c->off;
    const double* L0s = s->rest_len + c->off;
    const sf_membrane* m = &c->m;
    /* stretching (capsule.cpp:338-470) */
    for (int i = 0; i < n; ++i) {
        int j = nx_(c, i);
        v2 diff = min_image(c, NODE(c, j), NODE(c, i));
        double L = vnorm(diff);
        if (L < 1e-15) continue;
        double L0 = L0s[i];
        double F_mag;
        if (m->model == SF_NEO_HOOKEAN) {
            double lambda = L / L0;
            double lambda_inv3 = 1.0 / (lambda * lambda * lambda);
            F_mag = m->G_s * (lambda - lambda_inv3);
        } else if (m->model == SF_SKALAK) {
            double lambda = L / L0;
            double lambda2 = lambda * lambda;
            F_mag = m->G_s * lambda * (lambda2 - 1.0) * (1.0 + m->C_skalak);
        } else if (m->model == SF_WLC) {
            double L_max = m->wlc_L_max_ratio * L0;
            double x = L / L_max;
            if (x > 0.99) x = 0.99;
            double F_wlc = c->wlc_kBT_p * (1.0 / (4.0 * (1.0 - x) * (1.0 - x)) - 0.25 + x);
            double F_pow = -c->wlc_k_pow / L;
            F_mag = F_wlc + F_pow;
        } else {
            F_mag = m->k_stretch * (L / L0 - 1.0);
        }
        v2 dir = vdiv(diff, L);
        v2 Fe = vmul(dir, F_mag);
        F[i] = vadd(F[i], Fe);
        F[j] = vsub(F[j], Fe);
    }
    /* bending (capsule.cpp:476-541) */
    if (m->use_helfrich) {
        for (int i = 0; i < n; ++i) {
            const int ip = pv_(c, i), in = nx_(c, i);
            v2 e_prev = min_image(c, NODE(c, i), NODE(c, ip));
            v2 e_next = min_image(c, NODE(c, in), NODE(c, i));
            double lp2 = vdot(e_prev, e_prev), ln2 = vdot(e_next, e_next);
            if (lp2 < 1e-30 || ln2 < 1e-30) continue;
            double dth = atan2(vcross(e_prev, e_next), vdot(e_prev, e_next)) - s->rest_ang[c->off + i];
            double cc = -m->k_bend * dth / s->rest_ds[c->off + i];
            v2 gn = {-e_next.y, e_next.x}; gn = vdiv(gn, ln2);
            v2 gp = {-e_prev.y, e_prev.x}; gp = vdiv(gp, lp2);
            F[in] = vadd(F[in], vmul(gn, cc));
            F[ip] = vadd(F[ip], vmul(gp, cc));
            F[i] = vsub(F[i], vmul(vadd(gn, gp), cc));
        }
    } else {
        for (int i = 0; i < n; ++i) {
            v2 dp = min_image(c, NODE(c, pv_(c, i)), NODE(c, i));
            v2 dn = min_image(c, NODE(c, nx_(c, i)), NODE(c, i));
            v2 lap = vadd(dp, dn);
            F[i] = vadd(F[i], vmul(lap, m->k_bend));
        }
    }
    /* area (capsule.cpp:547-586) */
    {
        double A = cap_area(s, c), A0 = c->rest_area;
        if (!(A0 < 1e-15)) {
            double coeff = -m->k_area * (A - A0) / A0;
            double sa = 0.0;
            if (c->periodic_nx > 0) {
                v2* uw = (v2*)malloc(sizeof(v2) * n);
                uw[0] = NODE(c, 0);
                for (int k = 1; k < n; ++k) uw[k] = vadd(uw[k - 1], min_image(c, NODE(c, k), NODE(c, k - 1)));
                for (int k = 0; k < n; ++k) sa += vcross(uw[k], uw[(k + 1) % n]);
                free(uw);
            } else {
                for (int k = 0; k < n; ++k) sa += vcross(NODE(c, k), NODE(c, nx_(c, k)));
            }
            double sign = (sa >= 0.0) ? 1.0 : -1.0;
            for (int i = 0; i < n; ++i) {
                v2 e_prev = min_image(c, NODE(c, i), NODE(c, pv_(c, i)));
                v2 e_next = min_image(c, NODE(c, nx_(c, i)), NODE(c, i));
                v2 np_ = {e_prev.y, -e_prev.x};
                v2 nn_ = {e_next.y, -e_next.x};
                v2 outward = vmul(vadd(np_, nn_), 0.5);
                double len = vnorm(outward);
                if (len < 1e-15) continue;
                outward = vmul(vdiv(outward, len), sign);
                F[i] = vadd(F[i], vmul(outward, coeff));
            }
        }
    }
    /* perimeter (capsule.cpp:588-604) */
    {
        double P = cap_perimeter(s, c), P0 = c->rest_perimeter;
        if (!(P0 < 1e-15)) {
            double coeff = -m->k_perimeter * (P - P0) / P0;
            for (int i = 0; i < n; ++i) {
                int j = nx_(c, i);
                v2 diff = min_image(c, NODE(c, j), NODE(c, i));
                double L = vnorm(diff);
                if (L < 1e-15) continue;
                v2 t = vdiv(diff, L);
                F[i] = vsub(F[i], vmul(t, coeff));
                F[j] = vadd(F[j], vmul(t, coeff));
            }
        }
    }
    /* lab-frame damping (capsule.cpp:606-610) */
    for (int i = 0; i < n; ++i) F[i] = vsub(F[i], vmul(V[i], m->gamma_visc));
    /* Kelvin-Voigt (capsule.cpp:612-671) */
    if (m->eta_membrane > 0.0) {
        double* Lp = s->prev_len + c->off;
        if (!c->has_prev) {
            for (int i = 0; i < n; ++i) Lp[i] = vnorm(min_image(c, NODE(c, nx_(c, i)), NODE(c, i)));
            c->has_prev = 1;
        } else {
            for (int i = 0; i < n; ++i) {
                int j = nx_(c, i);
                v2 diff = min_image(c, NODE(c, j), NODE(c, i));
                double L = vnorm(diff);
                if (L < 1e-15) continue;
                double strain_rate = (L - Lp[i]) / L0s[i];
                double F_visc = m->eta_membrane * strain_rate;
                v2 Fe = vmul(vdiv(diff, L), F_visc);
                F[i] = vadd(F[i], Fe);
                F[j] = vsub(F[j], Fe);
                Lp[i] = L;
            }
        }
    }
}

void sfo_compute_membrane_forces(sfo_sim* s) {
    for (int c = 0; c < s->ncaps; ++c) membrane_forces(s, &s->caps[c]);
}

/* ------------------------------------------------------------------ */
/* Contact (reference repulsion.cpp:6-284, cell_list.h:36-146)         */
/* ------------------------------------------------------------------ */

static v2 pair_force(const sfo_sim* s, v2 pa, v2 va, v2 pb, v2 vb) {
    const sf_params* p = &s->p;
    const double Lx = (double)s->nx;
    v2 diff = vsub(pa, pb);
    if (Lx > 0.0) {
        if (diff.x > 0.5 * Lx) diff.x -= Lx;
        if (diff.x < -0.5 * Lx) diff.x += Lx;
    }
    double r = vnorm(diff);
    v2 zero = {0.0, 0.0};
    if (r < 1e-15 || r >= p->rep_r_cut) return zero;
    v2 nrm = vdiv(diff, r);
    double F_rep = p->rep_epsilon * pow(p->rep_sigma / r, (double)p->rep_power);
    double F_n = F_rep;
    v2 F_t = zero;
    if (p->rep_damping_normal > 0.0 || p->rep_friction > 0.0) {
        v2 vr = vsub(va, vb);
        double v_n = vr.x * nrm.x + vr.y * nrm.y;
        F_n = F_rep - p->rep_damping_normal * v_n;
        if (F_n < 0.0) F_n = 0.0;
        if (p->rep_friction > 0.0) {
            v2 vt = vsub(vr, vmul(nrm, v_n));
            double vtm = vnorm(vt);
            if (vtm > 1e-12) F_t = vmul(vdiv(vt, vtm), -p->rep_friction * F_n);
        }
    }
    return vadd(vmul(nrm, F_n), F_t);
}

/* Obstacle::signedDistance / normalAt of CircleObstacle and RectObstacle
 * (geometry/circle_obstacle.h:17-37, rect_obstacle.h:18-59); std::min and
 * std::max over initializer lists keep the first extremum. */
static double first_max3(double a, double b, double c) {
    double m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    return m;
}
static double first_min4(double a, double b, double c, double d) {
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    if (d < m) m = d;
    return m;
}
static double obstacle_sd(const obstacle_t* o, double x, double y) {
    if (!o->rect) {
        double dx = x - o->a, dy = y - o->b;
        return sqrt(dx * dx + dy * dy) - o->c;
    }
    double dx = first_max3(o->a - x, x - o->c, 0.0);
    double dy = first_max3(o->b - y, y - o->d, 0.0);
    double outside = sqrt(dx * dx + dy * dy);
    if (outside > 1e-15) return outside;
    return -first_min4(x - o->a, o->c - x, y - o->b, o->d - y);
}
static v2 obstacle_normal(const obstacle_t* o, double x, double y) {
    if (!o->rect) {
        double dx = x - o->a, dy = y - o->b;
        double d = sqrt(dx * dx + dy * dy);
        v2 e = {1.0, 0.0};
        if (d < 1e-15) return e;
        v2 n = {dx / d, dy / d};
        return n;
    }
    const double x0 = o->a, y0 = o->b, x1 = o->c, y1 = o->d;
    double cx = x < x0 ? x0 : (x1 < x ? x1 : x);       /* std::clamp */
    double cy = y < y0 ? y0 : (y1 < y ? y1 : y);
    v2 np = {cx, cy};
    if (cx == x && cy == y) {
        double dl = x - x0, dr = x1 - x, db = y - y0, dt = y1 - y;
        double dmin = first_min4(dl, dr, db, dt);
        if (dmin == dl) { np.x = x0; np.y = y; }
        else if (dmin == dr) { np.x = x1; np.y = y; }
        else if (dmin == db) { np.x = x; np.y = y0; }
        else { np.x = x; np.y = y1; }
    }
    double dx = x - np.x, dy = y - np.y;
    double d = sqrt(dx * dx + dy * dy);
    v2 n;
    if (d < 1e-15) {
        double dl = fabs(x - x0), dr = fabs(x - x1), db = fabs(y - y0), dt = fabs(y - y1);
        double dmin = first_min4(dl, dr, db, dt);
        if (dmin == dl) { n.x = -1.0; n.y = 0.0; }
        else if (dmin == dr) { n.x = 1.0; n.y = 0.0; }
        else if (dmin == db) { n.x = 0.0; n.y = -1.0; }
        else { n.x = 0.0; n.y = 1.0; }
        return n;
    }
    n.x = dx / d; n.y = dy / d;
    return n;
}

/* RepulsionForce::computeObstacleRepulsion (membrane/repulsion.cpp:180-235)
 * for every obstacle of the channel builder in order, after the pair and
 * wall repulsion (engine/simulation.cpp:494-498). */
static void obstacle_repulsion(sfo_sim* s) {
    const sf_params* p = &s->p;
    for (int o = 0; o < s->nobs; ++o) {
        const obstacle_t* ob = &s->obs[o];
        for (int k = 0; k < s->M; ++k) {
            double sd = obstacle_sd(ob, s->pos[k].x, s->pos[k].y);
            if (sd >= p->rep_r_cut) continue;
            double r = fabs(sd);
            if (r < 1e-15) r = 1e-15;
            v2 nrm = obstacle_normal(ob, s->pos[k].x, s->pos[k].y);
            double F_rep = p->rep_epsilon * pow(p->rep_sigma / r, (double)p->rep_power);
            if (sd < 0.0) {
                s->frc[k] = vadd(s->frc[k], vmul(nrm, F_rep * 10.0));
                continue;
            }
            double F_n = F_rep;
            v2 F_t = {0.0, 0.0};
            if (p->rep_damping_normal > 0.0 || p->rep_friction > 0.0) {
                v2 v = s->vel[k];
                double v_n = v.x * nrm.x + v.y * nrm.y;
                F_n = F_rep - p->rep_damping_normal * v_n;
                if (F_n < 0.0) F_n = 0.0;
                if (p->rep_friction > 0.0) {
                    v2 vt = vsub(v, vmul(nrm, v_n));
                    double vtm = vnorm(vt);
                    if (vtm > 1e-12) F_t = vmul(vdiv(vt, vtm), -p->rep_friction * F_n);
                }
            }
            s->frc[k] = vadd(s->frc[k], vadd(vmul(nrm, F_n), F_t));
        }
    }
}

static void wall_repulsion(sfo_sim* s, const capsule_t* c, double yb, double yt) {
    v2 zero = {0.0, 0.0};
    for (int i = 0; i < c->n; ++i) {
        int k = c->off + i;
        v2 pb = {s->pos[k].x, yb}, pt = {s->pos[k].x, yt};
        s->frc[k] = vadd(s->frc[k], pair_force(s, s->pos[k], s->vel[k], pb, zero));
        s->frc[k] = vadd(s->frc[k], pair_force(s, s->pos[k], s->vel[k], pt, zero));
    }
}

static void record_pair(sfo_sim* s, int a, int b) {
    s->pair_count[a]++;
    if (s->pair_len == s->pair_cap) {
        s->pair_cap = s->pair_cap ? 2 * s->pair_cap : 1024;
        s->pair_list = (int*)realloc(s->pair_list, sizeof(int) * s->pair_cap);
    }
    s->pair_list[s->pair_len++] = b;
}

void sfo_compute_repulsion(sfo_sim* s) {
    const int ncaps = s->ncaps;
    if (ncaps == 0) return;
    const double yb = 0.5, yt = (double)s->ny - 1.5;     /* simulation.cpp:486-491 */
    const double Lx = (double)s->nx;                      /* periodic channel */
    const double r_cut = s->p.rep_r_cut;
    s->pair_count = (int*)realloc(s->pair_count, sizeof(int) * (s->M > 0 ? s->M : 1));
    memset(s->pair_count, 0, sizeof(int) * s->M);
    s->pair_len = 0;
    if (s->M > 100) {
        /* cell list (cell_list.h:36-87) */
        double x_extent = Lx, x_origin = 0.0;
        int ncx = (int)floor(x_extent / r_cut); if (ncx < 1) ncx = 1;
        int ncy = (int)floor((yt - yb) / r_cut); if (ncy < 1) ncy = 1;
        double dx = x_extent / (double)ncx, dy = (yt - yb) / (double)ncy;
        int tot = ncx * ncy;
        int* cell_of = (int*)malloc(sizeof(int) * s->M);
        int* cnt = (int*)calloc(tot + 1, sizeof(int));
        for (int k = 0; k < s->M; ++k) {
            v2 p = s->pos[k];
            int ci;
            if (isnan(p.x) || isnan(p.y) || isinf(p.x) || isinf(p.y)) ci = 0;
            else {
                double px = p.x - x_origin;
                px = fmod(px, Lx);
                if (px < 0.0) px += Lx;
                int cx = (int)floor(px / dx);
                int cy = (int)floor((p.y - yb) / dy);
                if (cx < 0) cx = 0;
                if (cx >= ncx) cx = ncx - 1;
                if (cy < 0) cy = 0;
                if (cy >= ncy) cy = ncy - 1;
                ci = cy * ncx + cx;
            }
            cell_of[k] = ci;
            cnt[ci + 1]++;
        }
        for (int i = 0; i < tot; ++i) cnt[i + 1] += cnt[i];
        int* list = (int*)malloc(sizeof(int) * (s->M > 0 ? s->M : 1));
        int* fill = (int*)malloc(sizeof(int) * tot);
        memcpy(fill, cnt, sizeof(int) * tot);
        for (int k = 0; k < s->M; ++k) list[fill[cell_of[k]]++] = k;   /* insertion order */
        int* cap_of = (int*)malloc(sizeof(int) * (s->M > 0 ? s->M : 1));
        for (int c = 0; c < ncaps; ++c)
            for (int i = 0; i < s->caps[c].n; ++i) cap_of[s->caps[c].off + i] = c;
        for (int c = 0; c < ncaps; ++c) {
            const capsule_t* cp = &s->caps[c];
            for (int a = 0; a < cp->n; ++a) {
                int ka = cp->off + a;
                int ci = cell_of[ka];
                int cx = ci % ncx, cy = ci / ncx;
                for (int ddy = -1; ddy <= 1; ++ddy) {                /* cell_list.h:102-120 */
                    int yy = cy + ddy;
                    if (yy < 0 || yy >= ncy) continue;
                    for (int ddx = -1; ddx <= 1; ++ddx) {
                        int xx = cx + ddx;
                        if (xx < 0) xx += ncx;
                        if (xx >= ncx) xx -= ncx;
                        int cell = yy * ncx + xx;
                        for (int e = cnt[cell]; e < cnt[cell + 1]; ++e) {
                            int kb = list[e];
                            if (cap_of[kb] == c) continue;
                            record_pair(s, ka, kb);
                            s->frc[ka] = vadd(s->frc[ka], pair_force(s, s->pos[ka], s->vel[ka], s->pos[kb], s->vel[kb]));
                        }
                    }
                }
            }
            wall_repulsion(s, cp, yb, yt);
        }
        free(cell_of); free(cnt); free(list); free(fill); free(cap_of);
    } else {
        /* one-sided all pairs (repulsion.cpp:206-216) */
        for (int i = 0; i < ncaps; ++i) {
            const capsule_t* ci = &s->caps[i];
            for (int j = 0; j < ncaps; ++j) {
                if (i == j) continue;
                const capsule_t* cj = &s->caps[j];
                for (int a = 0; a < ci->n; ++a)
                    for (int b = 0; b < cj->n; ++b) {
                        int ka = ci->off + a, kb = cj->off + b;
                        record_pair(s, ka, kb);
                        s->frc[ka] = vadd(s->frc[ka], pair_force(s, s->pos[ka], s->vel[ka], s->pos[kb], s->vel[kb]));
                    }
            }
            wall_repulsion(s, ci, yb, yt);
        }
    }
}

int sfo_contact_pairs(const sfo_sim* s, int* counts, int* list, int list_cap) {
    if (counts) memcpy(counts, s->pair_count, sizeof(int) * s->M);
    int n = s->pair_len < list_cap ? s->pair_len : list_cap;
    if (list && n > 0) memcpy(list, s->pair_list, sizeof(int) * n);
    return s->pair_len;
}

/* ------------------------------------------------------------------ */
/* IBM (reference immersed_boundary.cpp:25-286)                        */
/* ------------------------------------------------------------------ */

static double min_image_ds(v2 a, v2 b, double Lx) {
    v2 d = vsub(a, b);
    if (Lx > 0.0) {
        if (d.x > 0.5 * Lx) d.x -= Lx;
        if (d.x < -0.5 * Lx) d.x += Lx;
    }
    return vnorm(d);
}

static double node_ds(const sfo_sim* s, const capsule_t* c, int k) {
    const double Lx = (double)s->nx;
    int kp = (k - 1 + c->n) % c->n, kn = (k + 1) % c->n;
    double dp = min_image_ds(NODE(c, k), NODE(c, kp), Lx);
    double dn = min_image_ds(NODE(c, kn), NODE(c, k), Lx);
    return 0.5 * (dp + dn);
}

static void spread_node(sfo_sim* s, v2 pos, v2 force, double ds) {
    if (isnan(pos.x) || isnan(pos.y) || isinf(pos.x) || isinf(pos.y)) return;
    if (isnan(force.x) || isnan(force.y)) return;
    const int nx = s->nx, ny = s->ny;
    int ix0 = (int)floor(pos.x), iy0 = (int)floor(pos.y);
    if (iy0 < -2 || iy0 >= ny + 2) return;
    for (int iy = iy0 - 1; iy <= iy0 + 2; ++iy) {
        for (int ix = ix0 - 1; ix <= ix0 + 2; ++ix) {
            int jx = ix;
            if (jx < 0) jx += nx;
            if (jx >= nx) jx -= nx;
            int jy = iy;
            if (jy < 0 || jy >= ny) continue;
            double rx = pos.x - (double)ix, ry = pos.y - (double)iy;
            double w = phi_tab(s->phi_tbl, rx) * phi_tab(s->phi_tbl, ry);
            if (w > 1e-15) {
                int n = jy * nx + jx;
                s->Fx[n] += force.x * w * ds;
                s->Fy[n] += force.y * w * ds;
            }
        }
    }
}

static v2 interp_point(const sfo_sim* s, v2 pos) {
    v2 u = {0.0, 0.0};
    if (isnan(pos.x) || isnan(pos.y) || isinf(pos.x) || isinf(pos.y)) return u;
    const int nx = s->nx, ny = s->ny;
    int ix0 = (int)floor(pos.x), iy0 = (int)floor(pos.y);
    if (iy0 < -2 || iy0 >= ny + 2) return u;
    for (int iy = iy0 - 1; iy <= iy0 + 2; ++iy) {
        for (int ix = ix0 - 1; ix <= ix0 + 2; ++ix) {
            int jx = ix;
            if (jx < 0) jx += nx;
            if (jx >= nx) jx -= nx;
            int jy = iy;
            if (jy < 0 || jy >= ny) continue;
            double rx = pos.x - (double)ix, ry = pos.y - (double)iy;
            double w = phi_tab(s->phi_tbl, rx) * phi_tab(s->phi_tbl, ry);
            if (w > 1e-15) {
                int n = jy * nx + jx;
                u.x += s->ux[n] * w;
                u.y += s->uy[n] * w;
            }
        }
    }
    return u;
}

void sfo_spread_forces(sfo_sim* s) {
    for (int c = 0; c < s->ncaps; ++c) {
        const capsule_t* cp = &s->caps[c];
        for (int k = 0; k < cp->n; ++k)
            spread_node(s, NODE(cp, k), s->frc[cp->off + k], node_ds(s, cp, k));
    }
}

/* reference immersed_boundary.cpp:231-286 */
static void multi_direct_forcing(sfo_sim* s, int K) {
    sfo_spread_forces(s);
    if (K <= 1) return;
    for (int it = 1; it < K; ++it) {
        sfo_compute_macroscopic(s);
        for (int c = 0; c < s->ncaps; ++c) {
            const capsule_t* cp = &s->caps[c];
            for (int k = 0; k < cp->n; ++k) {
                v2 pos = NODE(cp, k);
                v2 ui = interp_point(s, pos);
                v2 ud = s->vel[cp->off + k];
                v2 du = vsub(ud, ui);
                double rho_local = 1.0;
                int ix = (int)(pos.x + 0.5), iy = (int)(pos.y + 0.5);
                if (ix < 0) ix += s->nx;
                if (ix >= s->nx) ix -= s->nx;
                if (iy >= 0 && iy < s->ny) rho_local = s->rho[iy * s->nx + ix];
                v2 dF = vmul(du, 2.0 * rho_local);
                spread_node(s, pos, dF, node_ds(s, cp, k));
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Engine (reference simulation.cpp:429-801)                           */
/* ------------------------------------------------------------------ */

void sfo_initialize(sfo_sim* s) {
    const int nx = s->nx, ny = s->ny, N = s->N;
    /* lbm_solver.cpp:130-170 */
    for (int n = 0; n < N; ++n) s->flags[n] = CT_FLUID;
    /* ChannelBuilder::applyToField (channel_builder.cpp:6-36): pillars */
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            for (int k = 0; k < s->nobs; ++k)
                if (obstacle_contains(&s->obs[k], (double)x, (double)y)) {
                    s->flags[y * nx + x] = CT_SOLID;
                    break;
                }
    for (int x = 0; x < nx; ++x) { s->flags[x] = CT_SOLID; s->flags[(ny - 1) * nx + x] = CT_SOLID; }
    if (s->p.boundary_type == BT_INLET_OUTLET) {
        for (int y = 1; y < ny - 1; ++y) {
            s->flags[y * nx] = CT_INLET;
            s->flags[y * nx + nx - 1] = CT_OUTLET;
        }
    } else if (s->p.boundary_type == BT_CLOSED) {
        for (int y = 0; y < ny; ++y) { s->flags[y * nx] = CT_SOLID; s->flags[y * nx + nx - 1] = CT_SOLID; }
    }
    if (s->p.periodic_y) {
        for (int x = 0; x < nx; ++x) { s->flags[x] = CT_FLUID; s->flags[(ny - 1) * nx + x] = CT_FLUID; }
    }
    for (int n = 0; n < N; ++n) {
        s->rho[n] = s->p.rho0; s->ux[n] = 0.0; s->uy[n] = 0.0;
        for (int q = 0; q < Q; ++q) s->f[q * N + n] = feq(q, s->p.rho0, 0.0, 0.0);
    }
    memset(s->Fx, 0, sizeof(double) * N);
    memset(s->Fy, 0, sizeof(double) * N);
    sfo_compute_macroscopic(s);
    /* simulation.cpp:439-442: links only with a channel builder */
    s->nlinks = 0;
    if (s->nobs > 0 && s->p.use_interpolated_bb) ibb_build(s);
    /* advection_diffusion.cpp:46-57 with initial concentration 0 */
    memset(s->g, 0, sizeof(double) * N * Q);
    memset(s->C, 0, sizeof(double) * N);
}

static void one_step(sfo_sim* s) {
    const int N = s->N;
    memset(s->Fx, 0, sizeof(double) * N);                     /* step 0 */
    memset(s->Fy, 0, sizeof(double) * N);
    for (int k = 0; k < s->M; ++k) { s->frc[k].x = 0.0; s->frc[k].y = 0.0; }   /* 1 */
    sfo_compute_membrane_forces(s);                           /* 2 */
    sfo_compute_repulsion(s);                                 /* 3 */
    obstacle_repulsion(s);
    /* 4: with K > 1 the macroscopic recompute runs even without capsules */
    if (s->p.ibm_iterations > 1) multi_direct_forcing(s, s->p.ibm_iterations);
    else sfo_spread_forces(s);
    {                                                         /* 5: simulation.cpp:540-572 */
        const double bfx = s->p.body_fx, bfy = s->p.body_fy;
        if (bfx != 0.0 || bfy != 0.0) {
            for (int n = 0; n < N; ++n)
                if (s->flags[n] == CT_FLUID) { s->Fx[n] += bfx; s->Fy[n] += bfy; }
        }
    }
    {                                                         /* 6b: simulation.cpp:588-609 */
        const double Fm = s->p.max_lattice_force, Fm2 = Fm * Fm;
        int capped = 0;
        for (int n = 0; n < N; ++n) {
            double fx = s->Fx[n], fy = s->Fy[n];
            double f2 = fx * fx + fy * fy;
            if (f2 > Fm2) {
                double sc = Fm / sqrt(f2);
                s->Fx[n] *= sc; s->Fy[n] *= sc;
                ++capped;
            }
        }
        s->last_capped = capped;
    }
    lbm_step(s);                                              /* 7 */
    if (s->p.scalar_enabled) { adr_step(s); chemistry(s); }  /* 7c */
    for (int c = 0; c < s->ncaps; ++c) {                      /* 8 */
        const capsule_t* cp = &s->caps[c];
        for (int k = 0; k < cp->n; ++k) s->vel[cp->off + k] = interp_point(s, NODE(cp, k));
    }
    for (int c = 0; c < s->ncaps; ++c) {                      /* 9: capsule.cpp:267-297 */
        const capsule_t* cp = &s->caps[c];
        const double Lx = (double)cp->periodic_nx;
        for (int k = 0; k < cp->n; ++k) {
            v2* p = &s->pos[cp->off + k];
            *p = vadd(*p, vmul(s->vel[cp->off + k], s->p.dt));
            if (cp->periodic_nx > 0) {
                while (p->x < 0.0) p->x += Lx;
                while (p->x >= Lx) p->x -= Lx;
            }
        }
    }
    if (!s->p.periodic_y) {                                   /* 10 */
        const double ymin = 1.5, ymax = (double)s->ny - 1.5;
        for (int k = 0; k < s->M; ++k) {
            if (s->pos[k].y < ymin) s->pos[k].y = ymin;
            if (s->pos[k].y > ymax) s->pos[k].y = ymax;
        }
    }
}

void sfo_step(sfo_sim* s, int nsteps) {
    for (int i = 0; i < nsteps; ++i) one_step(s);
}

/* ------------------------------------------------------------------ */
/* Accessors                                                           */
/* ------------------------------------------------------------------ */
int sfo_num_capsules(const sfo_sim* s) { return s->ncaps; }
int sfo_num_markers(const sfo_sim* s) { return s->M; }
const int* sfo_capsule_offsets(const sfo_sim* s) { return s->offsets; }
double* sfo_f(sfo_sim* s) { return s->f; }
double* sfo_rho(sfo_sim* s) { return s->rho; }
double* sfo_ux(sfo_sim* s) { return s->ux; }
double* sfo_uy(sfo_sim* s) { return s->uy; }
double* sfo_Fx(sfo_sim* s) { return s->Fx; }
double* sfo_Fy(sfo_sim* s) { return s->Fy; }
double* sfo_pos(sfo_sim* s) { return (double*)s->pos; }
double* sfo_vel(sfo_sim* s) { return (double*)s->vel; }
double* sfo_force(sfo_sim* s) { return (double*)s->frc; }
double* sfo_prev_len(sfo_sim* s) { return s->prev_len; }
double* sfo_g(sfo_sim* s) { return s->g; }
double* sfo_C(sfo_sim* s) { return s->C; }
int sfo_last_capped(const sfo_sim* s) { return s->last_capped; }
int sfo_has_prev(const sfo_sim* s, int c) { return s->caps[c].has_prev; }
double sfo_capsule_area(const sfo_sim* s, int c) { return cap_area(s, &s->caps[c]); }
double sfo_capsule_perimeter(const sfo_sim* s, int c) { return cap_perimeter(s, &s->caps[c]); }
double sfo_capsule_rest_area(const sfo_sim* s, int c) { return s->caps[c].rest_area; }
double sfo_capsule_deformation(const sfo_sim* s, int c) { return cap_deformation(s, &s->caps[c]); }
double sfo_capsule_inclination(const sfo_sim* s, int c) { return cap_inclination(s, &s->caps[c]); }
void sfo_capsule_centroid(const sfo_sim* s, int c, double* cx, double* cy) {
    v2 r = cap_centroid(s, &s->caps[c]);
    *cx = r.x; *cy = r.y;
}
