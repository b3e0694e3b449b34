// ref_ops.cpp -- harness around the reference's own drop program (TEST INFRASTRUCTURE ONLY).
//
// Built by oracle/Makefile into oracle/_ref/libref_ops.so from the reference sources where they lie
// (nothing of the reference is copied into this repository).  Imm_OPS.cpp is included with its
// `main` renamed so that every function of the reference library is available unchanged; the
// functions below set a case up the way Imm_OPS.cpp:65-202 does (with the radius and the initial
// profile as arguments instead of the compile-time constants RAIO_GOTA and ESPESSURA_INI) and
// replay the body of its step loop, Imm_OPS.cpp:252-287 and :368-371, call for call.
#define main itlbm_ref_imm_ops_main
#include "Imm_OPS.cpp"
#undef main

#include "../include/itlbm.h"

#include <unistd.h>

namespace {
struct RefOps {
    GEOMETRY geometry;
    PARAMETERS parameters;
    LATTICE lattice;
    OPERADOR op;
    CAMPOS_F campos;
    double *forca = nullptr;
    int n = 0;
    int steps = 0;
};
}  // namespace

extern "C" {

void *ref_ops_create(int nx, int ny, int tipo, double chi, double xi, double tau, double beta,
                     double A, double radius, double k_perfil, double v0, double rho_R,
                     double rho_B, int threads) {
    RefOps *r = new RefOps();
    r->op.tipo = tipo;
    r->op.chi = chi;
    r->op.xi = xi;
    r->op.nome = tipo == OP_P1 ? "P1" : tipo == OP_P3 ? "P3" : tipo == OP_F1 ? "F1"
                 : tipo == OP_F2 ? "F2" : "F3";
    GEOMETRY &g = r->geometry;
    g.nx = nx;
    g.ny = ny;
    g.nz = 1;
    g.ini = new int[nx * ny];
    for (int p = 0; p < nx * ny; p++) g.ini[p] = p + 1;  // read_geo numbering of an all-fluid box
    g.fluid = nx * ny;
    r->n = g.fluid;
    PARAMETERS &pa = r->parameters;
    pa.tau = tau;
    pa.tau_R = tau;
    pa.tau_B = tau;
    pa.tau_m = 1.0;
    pa.A_fact = A;
    pa.recoll = beta;
    pa.rho_ini_R = rho_R;
    pa.rho_ini_B = rho_B;
    pa.wett_R = 0.0;
    pa.n_threads = threads;
    if (threads > 0) omp_set_num_threads(threads);
    LATTICE &L = r->lattice;
    const int m = r->n * nvel;
    L.inif_R = new double[m];
    L.inif_R_new = new double[m];
    L.inif_B = new double[m];
    L.inif_B_new = new double[m];
    L.inif_m = new double[m];
    L.inif_m_new = new double[m];
    L.ini_stream = new int[m];
    L.ini_solid = new bool[m];
    if (r->op.forca()) {
        r->forca = new double[3 * r->n]();
        L.ini_force = r->forca;
    }
    L.c_i = new double[nvel * dim];
    def_lattice_d3q19(L);
    L.Q_i = new double[nvel * dim * dim];
    calc_Q(L);
    def_dir_prop(g, L);
    if (r->op.forca()) aloca_campos_F(r->campos, g, L);
    initial_conditions_drop(radius, k_perfil, 0.0, nx / 2, ny / 2, 0, v0, 0., 0., true, g, L, pa,
                            true, EQ_CLASSICO);
    for (int k = 0; k < m; k++) L.inif_R_new[k] = L.inif_B_new[k] = 0.0;
    return r;
}

void ref_ops_set_pops(void *h, const double *fR, const double *fB) {
    RefOps *r = (RefOps *)h;
    memcpy(r->lattice.inif_R, fR, sizeof(double) * r->n * nvel);
    memcpy(r->lattice.inif_B, fB, sizeof(double) * r->n * nvel);
}

void ref_ops_step(void *h, int nsteps) {
    RefOps *r = (RefOps *)h;
    LATTICE &lattice = r->lattice;
    PARAMETERS &parameters = r->parameters;
    OPERADOR &op = r->op;
    const int n_fluid = r->n;
    double *forca = r->forca;
    for (int s = 0; s < nsteps; s++) {
#pragma omp parallel for
        for (int pto = 0; pto < n_fluid; pto++) {
            const double rho_R = density(lattice.inif_R + pto * nvel);
            const double rho_B = density(lattice.inif_B + pto * nvel);
            emite_mediadores(lattice.inif_m + pto * nvel, (rho_R - rho_B) / (rho_R + rho_B), lattice);
            propag_site_med(lattice, parameters, pto);
        }
        {
            double *t = lattice.inif_m;
            lattice.inif_m = lattice.inif_m_new;
            lattice.inif_m_new = t;
        }
        if (op.forca()) calcula_forca(r->campos, op, parameters.A_fact, lattice, forca);
#pragma omp parallel for
        for (int pto = 0; pto < n_fluid; pto++) {
            static const double zero[3] = {0.0, 0.0, 0.0};
            const double *F = op.forca() ? forca + 3 * pto : zero;
            colisao_comum(lattice.inif_R + pto * nvel, lattice.inif_B + pto * nvel,
                          lattice.inif_m + pto * nvel, F, op, lattice, parameters);
            double mx = 0., my = 0., mz = 0.;
            propag_site(lattice, pto, mx, my, mz);
        }
        {
            double *t = lattice.inif_R;
            lattice.inif_R = lattice.inif_R_new;
            lattice.inif_R_new = t;
            t = lattice.inif_B;
            lattice.inif_B = lattice.inif_B_new;
            lattice.inif_B_new = t;
        }
        r->steps++;
    }
}

// which = 0: state at the top of the next step; which = 1: post-collision populations of the last
// step (after the swap they sit in the *_new arrays until the next push overwrites them).
void ref_ops_get_pops(void *h, int which, double *fR, double *fB) {
    RefOps *r = (RefOps *)h;
    const double *a = which ? r->lattice.inif_R_new : r->lattice.inif_R;
    const double *b = which ? r->lattice.inif_B_new : r->lattice.inif_B;
    memcpy(fR, a, sizeof(double) * r->n * nvel);
    memcpy(fB, b, sizeof(double) * r->n * nvel);
}

void ref_ops_get_force(void *h, double *F) {
    RefOps *r = (RefOps *)h;
    if (r->forca) memcpy(F, r->forca, sizeof(double) * 3 * r->n);
    else memset(F, 0, sizeof(double) * 3 * r->n);
}

// The diagnostic block Imm_OPS.cpp:293-304 on the post-collision populations of the last step.
int ref_ops_diag(void *h, int step, double v0, double x_ini, double y_ini, itlbm_drop_diag *out) {
    RefOps *r = (RefOps *)h;
    LATTICE L = r->lattice;
    std::swap(L.inif_R, L.inif_R_new);
    std::swap(L.inif_B, L.inif_B_new);
    DROP drop;
    drop.cilindro = true;
    drop.frac_in = FRAC_INTERNA;
    drop.frac_out = FRAC_EXTERNA;
    drop.espessura = ESPESSURA_INI;
    GI_DATA gi;
    const bool ok = calc_galilean(r->geometry, L, drop, gi, v0, step, x_ini, y_ini);
    if (ok) calc_perfil_logistico(r->geometry, L, drop);
    MODOS md;
    if (ok) md = modos_interface(r->geometry, L, drop.x0, drop.y0, drop.raio);
    memset(out, 0, sizeof(*out));
    out->ok = ok;
    out->step = step;
    out->x0 = drop.x0; out->y0 = drop.y0; out->area = drop.area; out->raio = drop.raio;
    out->raio_grad = drop.raio_grad; out->raio_linha = drop.raio_linha;
    out->massa_R = drop.massa_R; out->massa_B = drop.massa_B;
    out->qx = drop.qx; out->qy = drop.qy; out->qz = drop.qz;
    out->u_max = drop.u_max; out->u_rms = drop.u_rms;
    out->p_in = drop.p_in; out->p_out = drop.p_out; out->sd_in = drop.sd_in; out->sd_out = drop.sd_out;
    out->delta_p = drop.delta_p; out->sigma = drop.sigma; out->p_centro = drop.p_centro;
    out->p_canto = drop.p_canto; out->sigma_linha = drop.sigma_linha;
    out->K_perfil = drop.K_perfil; out->r_perfil = drop.r_perfil; out->res_perfil = drop.res_perfil;
    out->esp_perfil = drop.esp_perfil; out->n_perfil = drop.n_perfil;
    out->n_in = drop.n_in; out->n_out = drop.n_out; out->n_fluid = drop.n_fluid; out->n_ruim = drop.n_ruim;
    out->mean_x = gi.mean_x; out->mean_y = gi.mean_y; out->mean_z = gi.mean_z;
    out->drop_x = gi.drop_x; out->drop_y = gi.drop_y;
    out->max_ref = gi.max_ref; out->rms_ref = gi.rms_ref; out->max_mean = gi.max_mean;
    out->rms_mean = gi.rms_mean; out->max_lab = gi.max_lab; out->rms_lab = gi.rms_lab;
    out->min_f = gi.min_f; out->min_rho = gi.min_rho; out->min_phi = gi.min_phi; out->max_phi = gi.max_phi;
    out->axis_ratio = gi.axis_ratio; out->center_dx = gi.center_dx; out->center_dy = gi.center_dy;
    out->x_unwrapped = gi.x_unwrapped;
    out->negative_total = gi.negative_total; out->negative_color = gi.negative_color; out->bad = gi.bad;
    out->R0 = md.R0; out->a2 = md.a2; out->a4 = md.a4; out->a8 = md.a8; out->rmin = md.rmin; out->rmax = md.rmax;
    return ok ? 1 : 0;
}

// The final-field writers of Imm_OPS.cpp:357-364 (rec_density, rec_velocity) on the post-collision
// populations of the last step, run in directory `dir` (they write into the working directory).
int ref_ops_write_fields(void *h, int step, const char *dir) {
    RefOps *r = (RefOps *)h;
    LATTICE L = r->lattice;
    std::swap(L.inif_R, L.inif_R_new);
    std::swap(L.inif_B, L.inif_B_new);
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0) return 0;
    rec_density("rho_R", r->geometry, L.inif_R, (unsigned int)step);
    rec_density("rho_B", r->geometry, L.inif_B, (unsigned int)step);
    rec_velocity(r->geometry, L, (unsigned int)step);
    return chdir(cwd) == 0 ? 1 : 0;
}

void ref_ops_destroy(void *h) {
    RefOps *r = (RefOps *)h;
    LATTICE &L = r->lattice;
    delete[] L.inif_R; delete[] L.inif_R_new; delete[] L.inif_B; delete[] L.inif_B_new;
    delete[] L.inif_m; delete[] L.inif_m_new; delete[] L.ini_stream; delete[] L.ini_solid;
    delete[] L.c_i; delete[] L.Q_i;
    delete[] r->forca;
    delete[] r->geometry.ini;
    if (r->campos.viz) {
        delete[] r->campos.viz; delete[] r->campos.fase; delete[] r->campos.g; delete[] r->campos.aux;
    }
    delete r;
}

}  // extern "C"
