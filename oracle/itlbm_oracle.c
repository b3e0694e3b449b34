/*
 * itlbm_oracle.c -- CPU oracle of the colour-gradient LBM step (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C restatement of the reference's algorithm for the Imm_OPS / Imm_INCL stepping loop.  It
 * is the checker of the CUDA path: tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py use it; no product code links or calls it.  Each function cites the reference file:line
 * it follows (paths relative to the reference project root).  Arithmetic is written in the same
 * operation order as the reference so that the two agree to round-off; the build uses
 * -ffp-contract=off so the results do not depend on the host CPU.
 *
 * The mediator populations of the reference (emite_mediadores + propag_site_med + momentum,
 * SimBoltz_Functions/LBM_functions.cpp:1287-1337, 1057-1087) are restated algebraically: after the
 * push, the mediator i at node x holds w_i * (rho^N(x - c_i) * 3), so their momentum is
 * sum_i c_i w_i * (rho^N(x - c_i) * 3), accumulated in the same i order.
 */
#include "itlbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NV 19
#define ORC_PI 3.14159265358979323846 /* M_PI */

/* D3Q19 velocities and weights: def_lattice_d3q19 (SimBoltz_Functions/LBM_functions.cpp:366-497) */
static const int CI[NV][3] = {
    {0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
    {1, 1, 0},   {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1},  {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {0, -1, -1}, {0, 1, 1},  {0, -1, 1}, {0, 1, -1}};
static double W[NV];
static const double CS2 = 1. / 3.;      /* lattice.c_s2 */
static const double ONE_OVER_CS2 = 3.;  /* lattice.one_over_c_s2 */

static void lattice_init(void) {
    static int done = 0;
    if (done) return;
    W[0] = 1. / 3.;
    for (int i = 1; i < 7; i++) W[i] = 1. / 18.;
    for (int i = 7; i < NV; i++) W[i] = 1. / 36.;
    done = 1;
}

struct orc_case {
    int nx, ny, n;
    int tipo;
    double chi, xi, tau, beta, A;
    double *fR, *fB;         /* state at the top of a step (inif_R / inif_B after the swap)  */
    double *fR_post, *fB_post; /* post-collision populations of the last step               */
    double *fR_new, *fB_new;
    double *fase, *g, *aux, *force, *gm;
    int has_step;
};

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* density: SimBoltz_Functions/LBM_functions.cpp:1582-1590 */
static inline double density(const double *f) {
    double rho = 0.0;
    for (int i = 0; i < NV; i++) rho = rho + f[i];
    return rho;
}

/* dot_product: LBM_functions.cpp:865-876 */
static inline double dot3(const double *a, const double *b) {
    double r = 0.0;
    r = r + a[0] * b[0];
    r = r + a[1] * b[1];
    r = r + a[2] * b[2];
    return r;
}

static inline void cvec(int i, double *c) {
    c[0] = CI[i][0];
    c[1] = CI[i][1];
    c[2] = CI[i][2];
}

/* calcula: LBM_functions.cpp:1100-1171 (3-D branch) */
static void calcula(const double *f, double *vx, double *vy, double *vz, double *rho) {
    double mx = 0.0, my = 0.0, mz = 0.0, r = 0.0;
    for (int i = 0; i < NV; i++) {
        r = r + f[i];
        mx = mx + CI[i][0] * f[i];
        my = my + CI[i][1] * f[i];
        mz = mz + CI[i][2] * f[i];
    }
    if (r) {
        double inv = 1.0 / (r);
        *vx = mx * inv;
        *vy = my * inv;
        *vz = mz * inv;
    } else {
        *vx = 0.;
        *vy = 0.;
        *vz = 0.;
    }
    *rho = r;
}

/* momentum: LBM_functions.cpp:1057-1087 */
static void momentum(const double *f, double *mx, double *my, double *mz) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = 0; i < NV; i++) {
        a = a + CI[i][0] * f[i];
        b = b + CI[i][1] * f[i];
        c = c + CI[i][2] * f[i];
    }
    *mx = a;
    *my = b;
    *mz = c;
}

/* dist_eq: LBM_functions.cpp:890-945 (3-D branch) */
static void dist_eq(double *feq, double vx, double vy, double vz, double rho) {
    double v[3] = {vx, vy, vz};
    double vquad = (vx * vx + vy * vy + vz * vz);
    for (int i = 0; i < NV; i++) {
        double c[3];
        cvec(i, c);
        double cv = dot3(c, v);
        feq[i] = W[i] * rho *
                 (1.0 + cv * ONE_OVER_CS2 + 0.5 * cv * cv * ONE_OVER_CS2 * ONE_OVER_CS2 -
                  0.5 * vquad * ONE_OVER_CS2);
    }
}

/* source (Guo): LBM_functions.cpp:1603-1673 (3-D branch) */
static void source(double Fx, double Fy, double Fz, double vx, double vy, double vz, double rho,
                   double tau, double *S) {
    (void)rho;
    double v[3] = {vx, vy, vz}, F[3] = {Fx, Fy, Fz};
    double factor = (1. - 1. / (2. * tau));
    double vF = dot3(F, v);
    for (int i = 0; i < NV; i++) {
        double c[3];
        cvec(i, c);
        double cF = dot3(c, F);
        double cv = dot3(c, v);
        S[i] = factor * W[i] * ONE_OVER_CS2 * (cF + ONE_OVER_CS2 * cF * cv - vF);
    }
}

/* coll_BGK: SimBoltz_Functions/Collision_operators.cpp:8-46 */
static void coll_BGK(double *f, double ax, double ay, double az, double tau) {
    double feq[NV], S[NV], vx, vy, vz, rho;
    double one_over_tau = 1.0 / tau;
    calcula(f, &vx, &vy, &vz, &rho);
    double vxa = vx + 0.5 * ax, vya = vy + 0.5 * ay, vza = vz + 0.5 * az;
    double Fx = ax * rho, Fy = ay * rho, Fz = az * rho;
    source(Fx, Fy, Fz, vxa, vya, vza, rho, tau, S);
    dist_eq(feq, vxa, vya, vza, rho);
    for (int i = 0; i < NV; i++) {
        double op = (feq[i] - f[i]) * one_over_tau;
        f[i] = f[i] + op + S[i];
    }
}

/* coef_B: Operadores_tensao.cpp:94-109 */
static inline double coef_B(int tipo, double chi, double c2, double w) {
    if (tipo == ITLBM_OP_P1) return w / 3.0;
    double den = 6.0 * chi + 24.0;
    if (c2 < 0.5) return -(2.0 + 2.0 * chi) / (3.0 * chi + 12.0);
    if (c2 < 1.5) return chi / den;
    return 1.0 / den;
}

/* perturbacao: Operadores_tensao.cpp:116-133 */
void orc_perturbacao(int tipo, double chi, double A, const double *g, double *f) {
    lattice_init();
    double mod2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (mod2 <= 1.0e-60 || A == 0.0) return;
    double mod = sqrt(mod2);
    for (int i = 0; i < NV; i++) {
        double c0 = CI[i][0], c1 = CI[i][1], c2 = CI[i][2];
        double cg = c0 * g[0] + c1 * g[1] + c2 * g[2];
        double cc = c0 * c0 + c1 * c1 + c2 * c2;
        f[i] += A * mod * (W[i] * cg * cg / mod2 - coef_B(tipo, chi, cc, W[i]));
    }
}

void orc_source(const double *F, const double *u, double rho, double tau, double *S) {
    lattice_init();
    source(F[0], F[1], F[2], u[0], u[1], u[2], rho, tau, S);
}

/* recolloring: LBM_functions.cpp:1713-1746 */
static void recolloring(const double *f, double *fR, double *fB, const double *grad, double mod,
                        double cR, double cB, double rho, double beta) {
    double fator = beta * cR * cB;
    double cos_phi = 0.;
    fR[0] = cR * f[0];
    fB[0] = cB * f[0];
    for (int i = 1; i < NV; i++) {
        double c[3];
        cvec(i, c);
        double c_2 = dot3(c, c);
        double prod = dot3(c, grad);
        if (mod) cos_phi = prod / (mod * sqrt(c_2));
        else cos_phi = 0.0;
        fR[i] = cR * f[i] - fator * W[i] * rho * cos_phi;
        fB[i] = cB * f[i] + fator * W[i] * rho * cos_phi;
    }
}

/* colisao_comum: Operadores_tensao.cpp:340-373.  gm is the mediator momentum (= -grad rho^N). */
static void colisao_comum(int tipo, double chi, double tau, double A, double beta, double *fR,
                          double *fB, const double *gm, const double *F) {
    double rho_R = density(fR), rho_B = density(fB);
    double rho = rho_R + rho_B;
    if (rho <= 1.0e-30) return;
    double cR = rho_R / rho, cB = 1.0 - cR;
    double mod = sqrt(gm[0] * gm[0] + gm[1] * gm[1] + gm[2] * gm[2]);
    double f[NV];
    for (int i = 0; i < NV; i++) f[i] = fR[i] + fB[i];
    if (tipo >= ITLBM_OP_F1) {
        coll_BGK(f, F[0] / rho, F[1] / rho, F[2] / rho, tau);
    } else {
        coll_BGK(f, 0.0, 0.0, 0.0, tau);
        orc_perturbacao(tipo, chi, A, gm, f);
    }
    recolloring(f, fR, fB, gm, mod, cR, cB, rho, beta);
}

void orc_colisao_comum(int tipo, double chi, double tau, double A_fact, double beta, double *fR,
                       double *fB, const double *gm, const double *F) {
    lattice_init();
    static const double zero[3] = {0, 0, 0};
    colisao_comum(tipo, chi, tau, A_fact, beta, fR, fB, gm, F ? F : zero);
}

static inline int wrap(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

/* neighbour x + c_i on the periodic all-fluid slab: aloca_campos_F (Operadores_tensao.cpp:149-182)
 * and def_dir_prop (SimBoltz_Functions/LBM_functions.cpp:679-852) both reduce to this. */
static inline int viz(int x, int y, int i, int nx, int ny) {
    return wrap(x + CI[i][0], nx) + nx * wrap(y + CI[i][1], ny);
}

/* calcula_forca: Operadores_tensao.cpp:202-332, given the rho^N field `fase` */
static void force_from_fase(int tipo, double xi, double sigma, int nx, int ny, const double *fase,
                            double *gbuf, double *aux, double *F) {
    const int n = nx * ny;
#pragma omp parallel for
    for (int p = 0; p < n; p++) {
        int x = p % nx, y = p / nx;
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int i = 1; i < NV; i++) {
            double ph = W[i] * fase[viz(x, y, i, nx, ny)];
            gx += ph * CI[i][0];
            gy += ph * CI[i][1];
            gz += ph * CI[i][2];
        }
        gbuf[3 * p + 0] = 3.0 * gx;
        gbuf[3 * p + 1] = 3.0 * gy;
        gbuf[3 * p + 2] = 3.0 * gz;
    }
    const double kf = 0.75 * sigma * xi;
    const double bf = 3.0 * sigma / (8.0 * xi);
#pragma omp parallel for
    for (int p = 0; p < n; p++) {
        int x = p % nx, y = p / nx;
        const double *g = gbuf + 3 * p;
        double *a = aux + 6 * p;
        double m = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        if (tipo == ITLBM_OP_F1) {
            double inv = (m > 1.0e-12) ? 1.0 / m : 0.0;
            a[0] = g[0] * inv;
            a[1] = g[1] * inv;
            a[2] = g[2] * inv;
        } else if (tipo == ITLBM_OP_F2) {
            double h = 0.5 * sigma;
            double inv = (m > 1.0e-30) ? 1.0 / m : 0.0;
            a[0] = h * (m - g[0] * g[0] * inv);
            a[1] = h * (m - g[1] * g[1] * inv);
            a[2] = h * (m - g[2] * g[2] * inv);
            a[3] = -h * g[0] * g[1] * inv;
            a[4] = -h * g[0] * g[2] * inv;
            a[5] = -h * g[1] * g[2] * inv;
        } else {
            double ph = fase[p];
            double lap = 0.0;
            for (int i = 1; i < NV; i++) lap += W[i] * (fase[viz(x, y, i, nx, ny)] - ph);
            lap *= 6.0;
            a[0] = 4.0 * bf * ph * (ph * ph - 1.0) - kf * lap;
        }
    }
#pragma omp parallel for
    for (int p = 0; p < n; p++) {
        int x = p % nx, y = p / nx;
        const double *g = gbuf + 3 * p;
        double *Fp = F + 3 * p;
        if (tipo == ITLBM_OP_F1) {
            /* div_iso: Operadores_tensao.cpp:187-200 */
            double d = 0.0;
            for (int i = 1; i < NV; i++) {
                const double *vv = aux + 6 * viz(x, y, i, nx, ny);
                d += W[i] * (CI[i][0] * vv[0] + CI[i][1] * vv[1] + CI[i][2] * vv[2]);
            }
            double kappa = -(3.0 * d);
            Fp[0] = 0.5 * sigma * kappa * g[0];
            Fp[1] = 0.5 * sigma * kappa * g[1];
            Fp[2] = 0.5 * sigma * kappa * g[2];
        } else if (tipo == ITLBM_OP_F2) {
            double Fx = 0.0, Fy = 0.0, Fz = 0.0;
            for (int i = 1; i < NV; i++) {
                const double *T = aux + 6 * viz(x, y, i, nx, ny);
                double w = W[i];
                double c0 = CI[i][0], c1 = CI[i][1], c2 = CI[i][2];
                Fx += w * (T[0] * c0 + T[3] * c1 + T[4] * c2);
                Fy += w * (T[3] * c0 + T[1] * c1 + T[5] * c2);
                Fz += w * (T[4] * c0 + T[5] * c1 + T[2] * c2);
            }
            Fp[0] = 3.0 * Fx;
            Fp[1] = 3.0 * Fy;
            Fp[2] = 3.0 * Fz;
        } else {
            double mu = aux[6 * p];
            Fp[0] = mu * g[0];
            Fp[1] = mu * g[1];
            Fp[2] = mu * g[2];
        }
    }
}

static void compute_fase(int n, const double *fR, const double *fB, double *fase) {
#pragma omp parallel for
    for (int p = 0; p < n; p++) {
        double rR = density(fR + (size_t)p * NV);
        double rB = density(fB + (size_t)p * NV);
        fase[p] = (rR - rB) / (rR + rB);
    }
}

void orc_calcula_forca(int tipo, double xi, double sigma, int nx, int ny, const double *fR,
                       const double *fB, double *F) {
    lattice_init();
    int n = nx * ny;
    double *fase = malloc(sizeof(double) * n);
    double *g = malloc(sizeof(double) * 3 * n);
    double *aux = malloc(sizeof(double) * 6 * n);
    compute_fase(n, fR, fB, fase);
    force_from_fase(tipo, xi, sigma, nx, ny, fase, g, aux, F);
    free(fase);
    free(g);
    free(aux);
}

orc_case *orc_create(int nx, int ny, int tipo, double chi, double xi, double tau, double beta,
                     double A_fact) {
    lattice_init();
    orc_case *c = calloc(1, sizeof(orc_case));
    c->nx = nx;
    c->ny = ny;
    c->n = nx * ny;
    c->tipo = tipo;
    c->chi = chi;
    c->xi = xi;
    c->tau = tau;
    c->beta = beta;
    c->A = A_fact;
    size_t m = (size_t)c->n * NV;
    c->fR = calloc(m, sizeof(double));
    c->fB = calloc(m, sizeof(double));
    c->fR_post = calloc(m, sizeof(double));
    c->fB_post = calloc(m, sizeof(double));
    c->fR_new = calloc(m, sizeof(double));
    c->fB_new = calloc(m, sizeof(double));
    c->fase = calloc(c->n, sizeof(double));
    c->g = calloc(3 * (size_t)c->n, sizeof(double));
    c->aux = calloc(6 * (size_t)c->n, sizeof(double));
    c->force = calloc(3 * (size_t)c->n, sizeof(double));
    c->gm = calloc(3 * (size_t)c->n, sizeof(double));
    return c;
}

void orc_destroy(orc_case *c) {
    if (!c) return;
    free(c->fR);
    free(c->fB);
    free(c->fR_post);
    free(c->fB_post);
    free(c->fR_new);
    free(c->fB_new);
    free(c->fase);
    free(c->g);
    free(c->aux);
    free(c->force);
    free(c->gm);
    free(c);
}

/* initial_conditions_drop (SimBoltz_Functions/Initial_conditions.cpp:37-169) with the centre
 * (nx/2, ny/2, 0), cilindro = true, delta_rho = 0 and EQ_CLASSICO, as called at Imm_OPS.cpp:199-202. */
void orc_init_drop(orc_case *c, double radius, double k_perfil, double v0, double rho_Ri,
                   double rho_Bi) {
    const int nx = c->nx, ny = c->ny;
    const int x0 = nx / 2, y0 = ny / 2;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            double dx = (double)(x - x0), dy = (double)(y - y0), dz = 0.0;
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            double phi;
            if (k_perfil > 0.0) {
                double arg = k_perfil * (r - radius);
                if (arg > 60.0) arg = 60.0;
                if (arg < -60.0) arg = -60.0;
                phi = 1.0 / (1.0 + exp(arg));
            } else
                phi = (r < radius) ? 1.0 : 0.0;
            double rho_tot = rho_Bi + phi * (rho_Ri - rho_Bi) + phi * 0.0;
            int pto = x + y * nx;
            double rR = phi * rho_tot, rB = (1.0 - phi) * rho_tot;
            dist_eq(c->fR + (size_t)pto * NV, v0, 0., 0., rR);
            dist_eq(c->fB + (size_t)pto * NV, v0, 0., 0., rB);
        }
    c->has_step = 0;
}

/* logistic strip: Imm_INCL.cpp:309-334 (N = nx = ny) */
void orc_init_strip(orc_case *c, int p, int q) {
    const int N = c->nx;
    const double m = sqrt((double)(p * p + q * q));
    const double k = 2.0 * log(9.0) / 3.45;
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++) {
            long long s = ((long long)p * x + (long long)q * y) % N;
            if (s < 0) s += N;
            double a1 = (double)s, a2 = 0.5 * N - s;
            double b1 = s - 0.5 * N, b2 = (double)(N - s);
            double dred = (2 * s < N) ? (a1 < a2 ? a1 : a2) / m : -(b1 < b2 ? b1 : b2) / m;
            double cR = 1.0 / (1.0 + exp(-k * dred));
            int pto = x + y * N;
            for (int i = 0; i < NV; i++) {
                c->fR[(size_t)pto * NV + i] = W[i] * cR;
                c->fB[(size_t)pto * NV + i] = W[i] * (1.0 - cR);
            }
        }
    c->has_step = 0;
}

void orc_set_pops(orc_case *c, const double *fR, const double *fB) {
    memcpy(c->fR, fR, sizeof(double) * NV * (size_t)c->n);
    memcpy(c->fB, fB, sizeof(double) * NV * (size_t)c->n);
}

void orc_get_pops(const orc_case *c, int which, double *fR, double *fB) {
    const double *a = which ? c->fR_post : c->fR, *b = which ? c->fB_post : c->fB;
    memcpy(fR, a, sizeof(double) * NV * (size_t)c->n);
    memcpy(fB, b, sizeof(double) * NV * (size_t)c->n);
}

void orc_get_force(const orc_case *c, double *F) {
    memcpy(F, c->force, sizeof(double) * 3 * (size_t)c->n);
}

void orc_get_gm(const orc_case *c, double *gm) {
    memcpy(gm, c->gm, sizeof(double) * 3 * (size_t)c->n);
}

/* One time step: the loop body Imm_OPS.cpp:252-287 / Imm_INCL.cpp:364-396, followed by the swap
 * Imm_OPS.cpp:368-371.  The post-collision populations (what the diagnostics read) are kept. */
void orc_step(orc_case *c, int nsteps) {
    const int nx = c->nx, ny = c->ny, n = c->n;
    const int forca = c->tipo >= ITLBM_OP_F1;
    for (int s = 0; s < nsteps; s++) {
        /* mediator phase: density + emite_mediadores argument, Imm_OPS.cpp:255-258 */
        compute_fase(n, c->fR, c->fB, c->fase);
        /* mediator momentum after propag_site_med: gm(x) = sum_i c_i * (w_i * (fase(x - c_i) * 3)) */
#pragma omp parallel for
        for (int p = 0; p < n; p++) {
            int x = p % nx, y = p / nx;
            double M[NV];
            for (int i = 0; i < NV; i++) {
                int src = wrap(x - CI[i][0], nx) + nx * wrap(y - CI[i][1], ny);
                double fat = c->fase[src] * ONE_OVER_CS2;
                M[i] = W[i] * fat;
            }
            momentum(M, &c->gm[3 * p], &c->gm[3 * p + 1], &c->gm[3 * p + 2]);
        }
        if (forca) force_from_fase(c->tipo, c->xi, c->A, nx, ny, c->fase, c->g, c->aux, c->force);
        /* colisao_comum + propag_site (push): Imm_OPS.cpp:275-287, LBM_functions.cpp:1220-1247 */
#pragma omp parallel for
        for (int p = 0; p < n; p++) {
            static const double zero[3] = {0, 0, 0};
            int x = p % nx, y = p / nx;
            double *fR = c->fR + (size_t)p * NV, *fB = c->fB + (size_t)p * NV;
            colisao_comum(c->tipo, c->chi, c->tau, c->A, c->beta, fR, fB, &c->gm[3 * p],
                          forca ? &c->force[3 * p] : zero);
            for (int i = 0; i < NV; i++) {
                size_t d = (size_t)viz(x, y, i, nx, ny) * NV + i;
                c->fR_new[d] = fR[i];
                c->fB_new[d] = fB[i];
            }
        }
        /* keep the post-collision arrays, then swap new -> current */
        double *t;
        t = c->fR_post; c->fR_post = c->fR; c->fR = c->fR_new; c->fR_new = t;
        t = c->fB_post; c->fB_post = c->fB; c->fB = c->fB_new; c->fB_new = t;
        c->has_step = 1;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* diagnostics of a drop                                                                      */
/* ------------------------------------------------------------------------------------------ */

static inline double gi_image(double dx, double length) {
    /* Galilean_diagnostics.cpp:18-20 */
    return dx - length * floor(dx / length + 0.5);
}

static inline int isfin(double v) { return isfinite(v); }

/* calc_drop_radius: SimBoltz_Functions/Other_functions.cpp:60-276 (cilindro, nz = 1) */
static void calc_drop_radius(const orc_case *c, const double *fR, const double *fB,
                             const double *force, itlbm_drop_diag *d) {
    const int nx = c->nx, ny = c->ny, nz = 1, nv = c->n;
    const double pi = 3.14159265358979323846;
    const double tx = 2.0 * pi / (double)nx, ty = 2.0 * pi / (double)ny, tz = 2.0 * pi / (double)nz;
    double massa_R = 0, massa_B = 0, qx = 0, qy = 0, qz = 0, area = 0, u2_sum = 0, u_max = 0;
    double cx_c = 0, cx_s = 0, cy_c = 0, cy_s = 0, cz_c = 0, cz_s = 0;
    int n_ruim = 0, n_fluid = 0;
    for (int pos = 0; pos < nv; pos++) {
        int pto = pos;
        double vxR, vyR, vzR, rho_R, vxB, vyB, vzB, rho_B;
        calcula(fR + (size_t)pto * NV, &vxR, &vyR, &vzR, &rho_R);
        calcula(fB + (size_t)pto * NV, &vxB, &vyB, &vzB, &rho_B);
        n_fluid = n_fluid + 1;
        if (!(rho_R == rho_R) || !(rho_B == rho_B) || !(vxR == vxR) || !(vxB == vxB)) {
            n_ruim = n_ruim + 1;
            continue;
        }
        massa_R = massa_R + rho_R;
        massa_B = massa_B + rho_B;
        qx = qx + rho_R * vxR + rho_B * vxB;
        qy = qy + rho_R * vyR + rho_B * vyB;
        qz = qz + rho_R * vzR + rho_B * vzB;
        double rho = rho_R + rho_B;
        if (rho <= 0.0) continue;
        double ux = (rho_R * vxR + rho_B * vxB) / rho;
        double uy = (rho_R * vyR + rho_B * vyB) / rho;
        double uz = (rho_R * vzR + rho_B * vzB) / rho;
        if (force) {
            const double *F = force + (size_t)pto * 3;
            ux = ux - 0.5 * F[0] / rho;
            uy = uy - 0.5 * F[1] / rho;
            uz = uz - 0.5 * F[2] / rho;
            qx = qx - 0.5 * F[0];
            qy = qy - 0.5 * F[1];
            qz = qz - 0.5 * F[2];
        }
        double u2 = ux * ux + uy * uy + uz * uz;
        u2_sum = u2_sum + u2;
        double u = sqrt(u2);
        if (u > u_max) u_max = u;
        double phi = rho_R / rho;
        area = area + phi;
        int z = pos / (nx * ny);
        int y = (pos - z * nx * ny) / nx;
        int x = pos - z * nx * ny - y * nx;
        cx_c = cx_c + phi * cos(tx * x);
        cx_s = cx_s + phi * sin(tx * x);
        cy_c = cy_c + phi * cos(ty * y);
        cy_s = cy_s + phi * sin(ty * y);
        cz_c = cz_c + phi * cos(tz * z);
        cz_s = cz_s + phi * sin(tz * z);
    }
    double x0 = atan2(cx_s, cx_c) / tx;
    if (x0 < 0.0) x0 += nx;
    double y0 = atan2(cy_s, cy_c) / ty;
    if (y0 < 0.0) y0 += ny;
    double z0 = 0.0; /* nz == 1 */
    (void)cz_c;
    (void)cz_s;
    double raio = (area > 0.0) ? sqrt(area / (pi * (double)nz)) : 0.0;

    double som_w = 0, som_wr = 0, sx_e = 0, sw_e = 0, sx_d = 0, sw_d = 0;
    int y_lin = (int)(y0 + 0.5);
    if (y_lin >= ny) y_lin -= ny;
    int z_lin = 0;
    for (int pos = 0; pos < nv; pos++) {
        double rho_R = density(fR + (size_t)pos * NV), rho_B = density(fB + (size_t)pos * NV);
        if (!(rho_R == rho_R) || !(rho_B == rho_B)) continue;
        int z = pos / (nx * ny);
        int y = (pos - z * nx * ny) / nx;
        int x = pos - z * nx * ny - y * nx;
        double dx = (double)x - x0;
        if (dx > 0.5 * nx) dx -= nx;
        if (dx < -0.5 * nx) dx += nx;
        double dy = (double)y - y0;
        if (dy > 0.5 * ny) dy -= ny;
        if (dy < -0.5 * ny) dy += ny;
        double dz = 0.0;
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double w = rho_R * rho_B;
        som_w = som_w + w;
        som_wr = som_wr + w * r;
        if (y == y_lin && z == z_lin) {
            if (dx < 0.0) {
                sx_e = sx_e + w * (double)x;
                sw_e = sw_e + w;
            } else {
                sx_d = sx_d + w * (double)x;
                sw_d = sw_d + w;
            }
        }
    }
    d->x0 = x0;
    d->y0 = y0;
    (void)z0;
    d->area = area;
    d->raio = raio;
    d->raio_grad = (som_w > 0.0) ? som_wr / som_w : 0.0;
    d->raio_linha = (sw_e > 0.0 && sw_d > 0.0) ? 0.5 * (sx_d / sw_d - sx_e / sw_e) : 0.0;
    d->massa_R = massa_R;
    d->massa_B = massa_B;
    d->qx = qx;
    d->qy = qy;
    d->qz = qz;
    d->u_max = u_max;
    d->u_rms = (n_fluid > 0) ? sqrt(u2_sum / (double)n_fluid) : 0.0;
    d->n_fluid = n_fluid;
    d->n_ruim = n_ruim;
}

/* calc_laplace_tension: Other_functions.cpp:453-554 with the DROP inputs of Imm_OPS.cpp:222-226 */
static void calc_laplace_tension(const orc_case *c, const double *fR, const double *fB,
                                 const double *force, itlbm_drop_diag *d) {
    calc_drop_radius(c, fR, fB, force, d);
    const int nx = c->nx, ny = c->ny, nv = c->n;
    const double frac_in = 0.5, frac_out = 2.0, espessura = 3.45;
    double x0 = d->x0, y0 = d->y0, raio = d->raio;
    double r_in_max = frac_in * raio;
    double r_out_min = frac_out * raio;
    if (r_out_min < raio + 4.0 * espessura) r_out_min = raio + 4.0 * espessura;
    double r_caixa = 0.45 * (double)((nx < ny) ? nx : ny);
    if (r_out_min > r_caixa) r_out_min = r_caixa;
    double p_in_s = 0, p_out_s = 0, p_in_s2 = 0, p_out_s2 = 0, p_ctr = 0, p_cnt = 0;
    int n_in = 0, n_out = 0, n_ctr = 0;
    for (int pos = 0; pos < nv; pos++) {
        double rho_R = density(fR + (size_t)pos * NV), rho_B = density(fB + (size_t)pos * NV);
        if (!(rho_R == rho_R) || !(rho_B == rho_B)) continue;
        int y = pos / nx, x = pos - y * nx;
        double dx = (double)x - x0;
        if (dx > 0.5 * nx) dx -= nx;
        if (dx < -0.5 * nx) dx += nx;
        double dy = (double)y - y0;
        if (dy > 0.5 * ny) dy -= ny;
        if (dy < -0.5 * ny) dy += ny;
        double dz = 0.0;
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double p = CS2 * (rho_R + rho_B);
        if (r < r_in_max) {
            p_in_s = p_in_s + p;
            p_in_s2 = p_in_s2 + p * p;
            n_in = n_in + 1;
        } else if (r >= r_out_min) {
            p_out_s = p_out_s + p;
            p_out_s2 = p_out_s2 + p * p;
            n_out = n_out + 1;
        }
        if (r < 1.5) {
            p_ctr = p_ctr + p;
            n_ctr = n_ctr + 1;
        }
        if (pos == 0) p_cnt = p_cnt + p;
    }
    double p_in = (n_in > 0) ? p_in_s / (double)n_in : 0.0;
    double p_out = (n_out > 0) ? p_out_s / (double)n_out : 0.0;
    double var_in = (n_in > 0) ? p_in_s2 / (double)n_in - p_in * p_in : 0.0;
    double var_out = (n_out > 0) ? p_out_s2 / (double)n_out - p_out * p_out : 0.0;
    double fator_forma = 1.0;
    d->p_in = p_in;
    d->sd_in = (var_in > 0.0) ? sqrt(var_in) : 0.0;
    d->p_out = p_out;
    d->sd_out = (var_out > 0.0) ? sqrt(var_out) : 0.0;
    d->n_in = n_in;
    d->n_out = n_out;
    d->delta_p = p_in - p_out;
    d->sigma = fator_forma * raio * d->delta_p;
    d->p_centro = (n_ctr > 0) ? p_ctr / (double)n_ctr : 0.0;
    d->p_canto = p_cnt;
    d->sigma_linha = fator_forma * d->raio_linha * (d->p_centro - d->p_canto);
}

/* calc_perfil_logistico: Other_functions.cpp:318-448 (radial, cilindro) */
static void calc_perfil_logistico(const orc_case *c, const double *fR, const double *fB,
                                  itlbm_drop_diag *d) {
    const double eps = 1.0e-30;
    const int nx = c->nx, ny = c->ny, nz = 1, nv = c->n;
    const double d_casca = 0.5;
    const int n_casca = (int)(sqrt((double)(nx * nx + ny * ny + nz * nz)) / d_casca) + 2;
    double *soma_phi = calloc(n_casca, sizeof(double));
    double *soma_n = calloc(n_casca, sizeof(double));
    const double x0 = d->x0, y0 = d->y0;
    for (int pos = 0; pos < nv; pos++) {
        double rho_R = density(fR + (size_t)pos * NV), rho_B = density(fB + (size_t)pos * NV);
        double rho = rho_R + rho_B;
        if (rho <= eps) continue;
        int y = pos / nx, x = pos - y * nx;
        double dx = (double)x - x0;
        if (dx > 0.5 * nx) dx -= nx;
        if (dx < -0.5 * nx) dx += nx;
        double dy = (double)y - y0;
        if (dy > 0.5 * ny) dy -= ny;
        if (dy < -0.5 * ny) dy += ny;
        double dz = 0.0;
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        int k = (int)(r / d_casca);
        if (k < 0 || k >= n_casca) continue;
        soma_phi[k] += rho_R / rho;
        soma_n[k] += 1.0;
    }
    double S = 0, Sr = 0, Sl = 0, Srr = 0, Srl = 0;
    int n_usadas = 0;
    for (int k = 0; k < n_casca; k++) {
        if (soma_n[k] < 1.0) continue;
        double phi = soma_phi[k] / soma_n[k];
        if (phi <= 0.02 || phi >= 0.98) continue;
        double r = ((double)k + 0.5) * d_casca;
        double l = log(phi / (1.0 - phi));
        S += 1.0;
        Sr += r;
        Sl += l;
        Srr += r * r;
        Srl += r * l;
        n_usadas++;
    }
    double K = 0.0, r_meio = 0.0, res_max = 0.0;
    if (n_usadas >= 3) {
        double den = S * Srr - Sr * Sr;
        if (fabs(den) > eps) {
            double a = (S * Srl - Sr * Sl) / den;
            double b = (Sl - a * Sr) / S;
            K = -a;
            if (fabs(a) > eps) r_meio = -b / a;
            for (int k = 0; k < n_casca; k++) {
                if (soma_n[k] < 1.0) continue;
                double phi = soma_phi[k] / soma_n[k];
                if (phi <= 0.02 || phi >= 0.98) continue;
                double r = ((double)k + 0.5) * d_casca;
                double dd = log(phi / (1.0 - phi)) - (a * r + b);
                if (fabs(dd) > res_max) res_max = fabs(dd);
            }
        }
    }
    free(soma_phi);
    free(soma_n);
    d->K_perfil = K;
    d->r_perfil = r_meio;
    d->res_perfil = res_max;
    d->esp_perfil = (K > eps) ? 2.0 * log(9.0) / K : 0.0;
    d->n_perfil = n_usadas;
}

/* modos_interface: Operadores_tensao.cpp:382-449 */
static double fase_em(const orc_case *c, const double *fR, const double *fB, double x, double y) {
    const int nx = c->nx, ny = c->ny;
    x = x - nx * floor(x / nx);
    y = y - ny * floor(y / ny);
    int i0 = (int)floor(x), j0 = (int)floor(y);
    double tx = x - i0, ty = y - j0;
    double v = 0.0;
    for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
            int ii = (i0 + di) % nx, jj = (j0 + dj) % ny;
            int p = ii + jj * nx;
            double rR = density(fR + (size_t)p * NV), rB = density(fB + (size_t)p * NV);
            double wgt = (di ? tx : 1 - tx) * (dj ? ty : 1 - ty);
            v += wgt * (rR - rB) / (rR + rB);
        }
    return v;
}

static void modos_interface(const orc_case *c, const double *fR, const double *fB, double x0,
                            double y0, double R_est, itlbm_drop_diag *d) {
    const int N_ANG = 256;
    double c2 = 0, s2 = 0, c4 = 0, s4 = 0, c8 = 0, s8 = 0, soma = 0;
    double rmin = 1e30, rmax = 0;
    for (int k = 0; k < N_ANG; k++) {
        double th = 2.0 * ORC_PI * k / N_ANG, ct = cos(th), st = sin(th);
        double a = 0.3 * R_est, b = 1.7 * R_est;
        double fa = fase_em(c, fR, fB, x0 + a * ct, y0 + a * st);
        for (int it = 0; it < 60; it++) {
            double mid = 0.5 * (a + b);
            double fm = fase_em(c, fR, fB, x0 + mid * ct, y0 + mid * st);
            if ((fm > 0) == (fa > 0)) a = mid;
            else b = mid;
        }
        double r = 0.5 * (a + b);
        soma += r;
        c2 += r * cos(2 * th);
        s2 += r * sin(2 * th);
        c4 += r * cos(4 * th);
        s4 += r * sin(4 * th);
        c8 += r * cos(8 * th);
        s8 += r * sin(8 * th);
        if (r < rmin) rmin = r;
        if (r > rmax) rmax = r;
    }
    d->R0 = soma / N_ANG;
    d->a2 = 2.0 * sqrt(c2 * c2 + s2 * s2) / N_ANG / d->R0;
    d->a4 = 2.0 * sqrt(c4 * c4 + s4 * s4) / N_ANG / d->R0;
    d->a8 = 2.0 * sqrt(c8 * c8 + s8 * s8) / N_ANG / d->R0;
    d->rmin = rmin;
    d->rmax = rmax;
}

/* calc_galilean (Galilean_diagnostics.cpp:24-105) then, when it succeeds, calc_perfil_logistico
 * and modos_interface: the diagnostic block Imm_OPS.cpp:299-304 on the post-collision state. */
int orc_diag_drop(orc_case *c, int step, double v0, double x_ini, double y_ini,
                  itlbm_drop_diag *d) {
    memset(d, 0, sizeof(*d));
    d->step = step;
    const int n = c->n, nx = c->nx, ny = c->ny;
    const double *fR = c->fR_post, *fB = c->fB_post;
    const double *force = (c->tipo >= ITLBM_OP_F1) ? c->force : NULL;
    double *ux = calloc(n, sizeof(double)), *uy = calloc(n, sizeof(double));
    double *uz = calloc(n, sizeof(double)), *ph = calloc(n, sizeof(double));
    d->min_f = INFINITY;
    d->min_rho = INFINITY;
    d->min_phi = 1;
    d->max_phi = 0;
    d->axis_ratio = 1;
    double mass = 0, mass_r = 0, qx = 0, qy = 0, qz = 0, qrx = 0, qry = 0;
    for (int p = 0; p < n; ++p) {
        double rr = 0, rb = 0, mx = 0, my = 0, mz = 0;
        for (int i = 0; i < NV; ++i) {
            double fr = fR[(size_t)p * NV + i], fb = fB[(size_t)p * NV + i];
            double f = fr + fb;
            if (!isfin(fr) || !isfin(fb)) ++d->bad;
            d->min_f = (f < d->min_f) ? f : d->min_f;
            if (f < -1.e-12) ++d->negative_total;
            if (fr < -1.e-12) ++d->negative_color;
            if (fb < -1.e-12) ++d->negative_color;
            rr += fr;
            rb += fb;
            mx += f * CI[i][0];
            my += f * CI[i][1];
            mz += f * CI[i][2];
        }
        double rho = rr + rb;
        if (!isfin(rho) || rho <= 0 || !isfin(mx) || !isfin(my) || !isfin(mz)) {
            ++d->bad;
            continue;
        }
        if (force) {
            const double *F = force + 3 * (size_t)p;
            if (!isfin(F[0]) || !isfin(F[1]) || !isfin(F[2])) {
                ++d->bad;
                continue;
            }
            mx -= 0.5 * F[0];
            my -= 0.5 * F[1];
            mz -= 0.5 * F[2];
        }
        d->min_rho = (rho < d->min_rho) ? rho : d->min_rho;
        ux[p] = mx / rho;
        uy[p] = my / rho;
        uz[p] = mz / rho;
        ph[p] = rr / rho;
        d->min_phi = (ph[p] < d->min_phi) ? ph[p] : d->min_phi;
        d->max_phi = (d->max_phi < ph[p]) ? ph[p] : d->max_phi;
        mass += rho;
        mass_r += rr;
        qx += mx;
        qy += my;
        qz += mz;
        qrx += rr * ux[p];
        qry += rr * uy[p];
    }
    int ok = 0;
    if (d->bad || !(mass > 0) || !(mass_r > 0)) goto done;
    d->mean_x = qx / mass;
    d->mean_y = qy / mass;
    d->mean_z = qz / mass;
    d->drop_x = qrx / mass_r;
    d->drop_y = qry / mass_r;
    calc_laplace_tension(c, fR, fB, force, d);
    {
        double sref = 0, smean = 0, slab = 0, sxx = 0, syy = 0, sxy = 0, sx = 0, sy = 0, weight = 0;
        double left_w = 0, right_w = 0, left_x = 0, right_x = 0;
        const int y_line = ((int)floor(d->y0 + 0.5)) % ny;
        for (int pos = 0; pos < nx * ny; ++pos) {
            int p = pos;
            double a = (ux[p] - v0) * (ux[p] - v0) + uy[p] * uy[p] + uz[p] * uz[p];
            double b = (ux[p] - d->mean_x) * (ux[p] - d->mean_x) +
                       (uy[p] - d->mean_y) * (uy[p] - d->mean_y) +
                       (uz[p] - d->mean_z) * (uz[p] - d->mean_z);
            double cc = ux[p] * ux[p] + uy[p] * uy[p] + uz[p] * uz[p];
            sref += a;
            smean += b;
            slab += cc;
            d->max_ref = fmax(d->max_ref, sqrt(a));
            d->max_mean = fmax(d->max_mean, sqrt(b));
            d->max_lab = fmax(d->max_lab, sqrt(cc));
            int x = pos % nx, y = pos / nx;
            double dx = gi_image(x - d->x0, nx), dy = gi_image(y - d->y0, ny), phi = ph[p];
            weight += phi;
            sx += phi * dx;
            sy += phi * dy;
            sxx += phi * dx * dx;
            syy += phi * dy * dy;
            sxy += phi * dx * dy;
            if (y == y_line) {
                double rr = density(fR + (size_t)p * NV), rb = density(fB + (size_t)p * NV);
                double w = rr * rb;
                if (dx < 0) {
                    left_w += w;
                    left_x += w * dx;
                } else {
                    right_w += w;
                    right_x += w * dx;
                }
            }
        }
        d->rms_ref = sqrt(sref / n);
        d->rms_mean = sqrt(smean / n);
        d->rms_lab = sqrt(slab / n);
        double xx = sxx / weight - (sx / weight) * (sx / weight);
        double yy = syy / weight - (sy / weight) * (sy / weight);
        double xy = sxy / weight - (sx / weight) * (sy / weight), trace = xx + yy;
        double disc = sqrt((xx - yy) * (xx - yy) + 4 * xy * xy);
        d->axis_ratio = (trace > disc) ? sqrt((trace + disc) / (trace - disc)) : INFINITY;
        d->center_dx = gi_image(d->x0 - (x_ini + v0 * step), nx);
        d->center_dy = gi_image(d->y0 - y_ini, ny);
        d->x_unwrapped = x_ini + v0 * step + d->center_dx;
        d->raio_linha = (left_w > 0 && right_w > 0) ? 0.5 * (right_x / right_w - left_x / left_w) : 0;
        int corner_x = ((int)floor(d->x0 + 0.5) + nx / 2) % nx;
        int corner_y = ((int)floor(d->y0 + 0.5) + ny / 2) % ny;
        int pc = corner_x + nx * corner_y;
        d->p_canto = density(fR + (size_t)pc * NV) * CS2 + density(fB + (size_t)pc * NV) * CS2;
        d->sigma_linha = d->raio_linha * (d->p_centro - d->p_canto);
        d->u_max = d->max_ref;
        d->u_rms = d->rms_ref;
        ok = isfin(d->sigma) && isfin(d->max_ref) && isfin(d->axis_ratio);
    }
    if (ok) {
        calc_perfil_logistico(c, fR, fB, d);
        modos_interface(c, fR, fB, d->x0, d->y0, d->raio, d);
    }
done:
    free(ux);
    free(uy);
    free(uz);
    free(ph);
    d->ok = ok;
    return ok;
}

/* ------------------------------------------------------------------------------------------ */
/* diagnostics of an inclined strip: mede_inclinada (Imm_INCL.cpp:74-189)                     */
/* ------------------------------------------------------------------------------------------ */

static double dist_central(int x, int y, int p, int q, int N) {
    double m = sqrt((double)(p * p + q * q));
    long long s = ((long long)p * x + (long long)q * y) % N;
    if (s < 0) s += N;
    double d = ((double)s - 0.5 * N);
    if (d >= 0.5 * N) d -= N;
    if (d < -0.5 * N) d += N;
    return -d / m;
}

int orc_diag_strip(orc_case *c, int step, int p, int q, itlbm_strip_diag *r) {
    memset(r, 0, sizeof(*r));
    r->step = step;
    r->min_f = 1e300;
    const int N = c->nx;
    const double *fRa = c->fR_post, *fBa = c->fB_post;
    const double *forca = (c->tipo >= ITLBM_OP_F1) ? c->force : NULL;
    const double m = sqrt((double)(p * p + q * q));
    const double nx_ = p / m, ny_ = q / m, tx_ = -ny_, ty_ = nx_;
    double u2 = 0, Sxx = 0, Sx = 0, Sxy = 0, Sy = 0;
    int nfit = 0;
    double *dd = malloc(sizeof(double) * (size_t)N * N), *ll = malloc(sizeof(double) * (size_t)N * N);
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++) {
            int pto = x + y * N;
            const double *fR = fRa + (size_t)pto * NV, *fB = fBa + (size_t)pto * NV;
            double rR = 0, rB = 0, jx = 0, jy = 0, Pxx = 0, Pyy = 0, Pxy = 0, Pzz = 0;
            for (int i = 0; i < NV; i++) {
                double c0 = CI[i][0], c1 = CI[i][1], c2 = CI[i][2];
                double f = fR[i] + fB[i];
                if (!isfin(fR[i]) || !isfin(fB[i])) r->n_ruim++;
                if (f < -1e-12) r->neg_total++;
                if (fR[i] < -1e-12) r->neg_cor++;
                if (fB[i] < -1e-12) r->neg_cor++;
                r->min_f = (f < r->min_f) ? f : r->min_f;
                rR += fR[i];
                rB += fB[i];
                jx += f * c0;
                jy += f * c1;
                Pxx += f * c0 * c0;
                Pyy += f * c1 * c1;
                Pxy += f * c0 * c1;
                Pzz += f * c2 * c2;
            }
            double rho = rR + rB;
            if (!(rho > 0)) {
                r->n_ruim++;
                continue;
            }
            if (forca) {
                jx -= 0.5 * forca[3 * pto];
                jy -= 0.5 * forca[3 * pto + 1];
                r->SFx += forca[3 * pto];
                r->SFy += forca[3 * pto + 1];
            }
            double ux = jx / rho, uy = jy / rho;
            r->massa_R += rR;
            r->massa_B += rB;
            r->qx += jx;
            r->qy += jy;
            double u = hypot(ux, uy), un = fabs(ux * nx_ + uy * ny_), ut = fabs(ux * tx_ + uy * ty_);
            r->u_max = fmax(r->u_max, u);
            r->un_max = fmax(r->un_max, un);
            r->ut_max = fmax(r->ut_max, ut);
            u2 += u * u;
            double Pnn = nx_ * nx_ * Pxx + 2 * nx_ * ny_ * Pxy + ny_ * ny_ * Pyy;
            double Ptt = tx_ * tx_ * Pxx + 2 * tx_ * ty_ * Pxy + ty_ * ty_ * Pyy;
            r->sigma_pop += Pnn - 0.5 * (Ptt + Pzz);
            const double *g = c->gm + 3 * (size_t)pto;
            r->int_grad += sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
            double d = dist_central(x, y, p, q, N);
            double cR = rR / rho;
            if (cR > 0.02 && cR < 0.98 && fabs(d) < 8.0) {
                double l = log(cR / (1.0 - cR));
                dd[nfit] = d;
                ll[nfit] = l;
                Sx += d;
                Sy += l;
                Sxx += d * d;
                Sxy += d * l;
                nfit++;
            }
        }
    double comprimento = 2.0 * N * m;
    r->sigma_pop /= comprimento;
    r->int_grad /= comprimento;
    r->u_rms = sqrt(u2 / (N * N));
    r->n_ajuste = nfit;
    if (nfit > 3) {
        double K = (nfit * Sxy - Sx * Sy) / (nfit * Sxx - Sx * Sx);
        double a = (Sy - K * Sx) / nfit;
        r->K = K;
        r->d0 = -a / K;
        for (int k = 0; k < nfit; k++) r->res = fmax(r->res, fabs(ll[k] - (a + K * dd[k])));
    }
    free(dd);
    free(ll);
    r->ok = (r->n_ruim == 0 && isfin(r->u_max));
    return r->ok;
}

/* ------------------------------------------------------------------------------------------ */
/* per-node output fields of the post-collision populations of the last step                  */
/* ------------------------------------------------------------------------------------------ */

/* form ITLBM_FIELDS_VTK: rec_density (LBM_functions.cpp:1457-1511) -- rho_R, rho_B by density() --
 * and rec_velocity's two-colour branch (:1349-1458): the colour velocities by calcula, weighted by the
 * concentrations, minus (F/2)/rho when the program keeps a force (class F, Imm_OPS.cpp:171-181).
 * form ITLBM_FIELDS_PROFILE: the columns of perfil.dat in mede_inclinada (Imm_INCL.cpp:104-162):
 * u = (sum_i f_i c_i - F/2) / rho with f_i = f_R,i + f_B,i; nodes with !(rho > 0) get no velocity
 * there (they are skipped), and NaN here. */
void orc_fields(const orc_case *c, int form, double *rho_R, double *rho_B, double *ux, double *uy,
                double *uz) {
    const double *forca = (c->tipo >= ITLBM_OP_F1) ? c->force : NULL;
    for (int p = 0; p < c->n; p++) {
        const double *fR = c->fR_post + (size_t)p * NV, *fB = c->fB_post + (size_t)p * NV;
        double rR = density(fR), rB = density(fB);
        double vx, vy, vz;
        if (form == ITLBM_FIELDS_VTK) {
            double vxR, vyR, vzR, rhoR, vxB, vyB, vzB, rhoB;
            calcula(fR, &vxR, &vyR, &vzR, &rhoR);
            calcula(fB, &vxB, &vyB, &vzB, &rhoB);
            double concR = rhoR / (rhoR + rhoB);
            double concB = 1. - concR;
            vx = concR * vxR + concB * vxB;
            vy = concR * vyR + concB * vyB;
            vz = concR * vzR + concB * vzB;
            if (forca) {
                double rho = rhoR + rhoB;
                const double *F = forca + 3 * (size_t)p;
                if (rho > 0.0) {
                    vx = vx - 0.5 * F[0] / rho;
                    vy = vy - 0.5 * F[1] / rho;
                    vz = vz - 0.5 * F[2] / rho;
                }
            }
        } else {
            double jx = 0, jy = 0, jz = 0;
            for (int i = 0; i < NV; i++) {
                double f = fR[i] + fB[i];
                jx += f * CI[i][0];
                jy += f * CI[i][1];
                jz += f * CI[i][2];
            }
            double rho = rR + rB;
            if (!(rho > 0)) {
                vx = vy = vz = NAN;
            } else {
                if (forca) {
                    jx -= 0.5 * forca[3 * (size_t)p];
                    jy -= 0.5 * forca[3 * (size_t)p + 1];
                    jz -= 0.5 * forca[3 * (size_t)p + 2];
                }
                vx = jx / rho;
                vy = jy / rho;
                vz = jz / rho;
            }
        }
        if (rho_R) rho_R[p] = rR;
        if (rho_B) rho_B[p] = rB;
        if (ux) ux[p] = vx;
        if (uy) uy[p] = vy;
        if (uz) uz[p] = vz;
    }
}
