/*
 * itlbm_oracle.h -- CPU oracle of the colour-gradient LBM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's algorithm for the
 * Imm_OPS / Imm_INCL stepping loop, used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py as the checker.  No product code links it or calls it.
 *
 * Parity of this restatement is pinned (tests/test_oracle_*.py) against
 *   - the reference itself, compiled from its sources into oracle/_ref/ by oracle/Makefile
 *     (population-level comparison after many steps, all seven operators), and
 *   - the reference's shipped golden outputs (Lotes/<batch>/<case>/laplace.dat, iso.dat,
 *     galilean.dat, inclinada.dat rows and E0_resultado.txt), committed under tests/golden/.
 *
 * Layout: populations in the reference's AoS order f[pto*19+i], pto = x + nx*y, nz = 1, all fluid.
 */
#ifndef ITLBM_ORACLE_H
#define ITLBM_ORACLE_H

#include "../include/itlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_case orc_case;

orc_case *orc_create(int nx, int ny, int tipo, double chi, double xi, double tau, double beta,
                     double A_fact);
void orc_destroy(orc_case *c);

void orc_init_drop(orc_case *c, double radius, double k_perfil, double v0, double rho_R,
                   double rho_B);
void orc_init_strip(orc_case *c, int p, int q);

void orc_set_pops(orc_case *c, const double *fR, const double *fB);
void orc_get_pops(const orc_case *c, int which, double *fR, double *fB);
void orc_get_force(const orc_case *c, double *F);
void orc_get_gm(const orc_case *c, double *gm);

void orc_step(orc_case *c, int nsteps);
void orc_set_threads(int n);

int orc_diag_drop(orc_case *c, int step, double v0, double x_ini, double y_ini,
                  itlbm_drop_diag *out);
int orc_diag_strip(orc_case *c, int step, int p, int q, itlbm_strip_diag *out);

/* per-node output fields of the post-collision populations of the last step; form is
 * ITLBM_FIELDS_VTK (rec_density / rec_velocity) or ITLBM_FIELDS_PROFILE (perfil.dat columns) */
void orc_fields(const orc_case *c, int form, double *rho_R, double *rho_B, double *ux, double *uy,
                double *uz);

/* per-site operator functions (E0 checks) */
void orc_perturbacao(int tipo, double chi, double A, const double *g, double *f);
void orc_source(const double *F, const double *u, double rho, double tau, double *S);
void orc_calcula_forca(int tipo, double xi, double sigma, int nx, int ny, const double *fR,
                       const double *fB, double *F);
void orc_colisao_comum(int tipo, double chi, double tau, double A_fact, double beta, double *fR,
                       double *fB, const double *gm, const double *F);

#ifdef __cplusplus
}
#endif

#endif
