// ref_incl.cpp -- harness around the reference's inclined-interface program (TEST INFRASTRUCTURE
// ONLY).  Built by oracle/Makefile into oracle/_ref/libref_incl.so from the reference sources where
// they lie.  Imm_INCL.cpp is included with its `main` renamed, which makes mede_inclinada
// (Imm_INCL.cpp:85-189) and the whole library available unchanged.  The set-up below follows
// Imm_INCL.cpp:192-334 and the step replays Imm_INCL.cpp:364-396 and :438-441 call for call.
#define main itlbm_ref_imm_incl_main
#include "Imm_INCL.cpp"
#undef main

#include "../include/itlbm.h"

#include <unistd.h>

namespace {
struct RefIncl {
    GEOMETRY geometry;
    PARAMETERS parameters;
    LATTICE lattice;
    OPERADOR op;
    CAMPOS_F campos;
    double *forca = nullptr;
    int n = 0, p = 1, q = 0;
};
}  // namespace

extern "C" {

void *ref_incl_create(int N, int tipo, double chi, double xi, double tau, double beta, double A,
                      int p, int q, int threads) {
    RefIncl *r = new RefIncl();
    r->op.tipo = tipo;
    r->op.chi = chi;
    r->op.xi = xi;
    r->p = p;
    r->q = q;
    GEOMETRY &g = r->geometry;
    g.nx = N;
    g.ny = N;
    g.nz = 1;
    g.ini = new int[N * N];
    for (int k = 0; k < N * N; k++) g.ini[k] = k + 1;
    g.fluid = N * N;
    r->n = g.fluid;
    PARAMETERS &pa = r->parameters;
    pa.tau = tau;
    pa.tau_R = tau;
    pa.tau_B = tau;
    pa.A_fact = A;
    pa.recoll = beta;
    pa.rho_ini_R = 1.0;
    pa.rho_ini_B = 1.0;
    pa.wett_R = 0.0;
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
    // the logistic strip of Imm_INCL.cpp:309-334
    const double mm = sqrt((double)(p * p + q * q));
    const double k = 2.0 * log(9.0) / ESPESSURA_INI;
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++) {
            long long s = ((long long)p * x + (long long)q * y) % N;
            if (s < 0) s += N;
            const double dred = (2 * s < N) ? min((double)s, 0.5 * N - s) / mm
                                            : -min(s - 0.5 * N, (double)(N - s)) / mm;
            const double cR = 1.0 / (1.0 + exp(-k * dred));
            const int pto = g.ini[x + y * N] - 1;
            for (int i = 0; i < nvel; i++) {
                L.inif_R[(size_t)pto * nvel + i] = L.w[i] * cR;
                L.inif_B[(size_t)pto * nvel + i] = L.w[i] * (1.0 - cR);
                L.inif_m[(size_t)pto * nvel + i] = 0.0;
            }
        }
    for (int kk = 0; kk < m; kk++) L.inif_R_new[kk] = L.inif_B_new[kk] = L.inif_m_new[kk] = 0.0;
    return r;
}

void ref_incl_step(void *h, int nsteps) {
    RefIncl *r = (RefIncl *)h;
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
    }
}

void ref_incl_get_pops(void *h, int which, double *fR, double *fB) {
    RefIncl *r = (RefIncl *)h;
    const double *a = which ? r->lattice.inif_R_new : r->lattice.inif_R;
    const double *b = which ? r->lattice.inif_B_new : r->lattice.inif_B;
    memcpy(fR, a, sizeof(double) * r->n * nvel);
    memcpy(fB, b, sizeof(double) * r->n * nvel);
}

// mede_inclinada (Imm_INCL.cpp:404) on the post-collision populations of the last step.
int ref_incl_diag(void *h, int step, itlbm_strip_diag *out) {
    RefIncl *r = (RefIncl *)h;
    LATTICE L = r->lattice;
    std::swap(L.inif_R, L.inif_R_new);
    std::swap(L.inif_B, L.inif_B_new);
    INCL res;
    const bool ok = mede_inclinada(r->geometry, L, r->p, r->q, res, r->forca, false);
    memset(out, 0, sizeof(*out));
    out->ok = ok;
    out->step = step;
    out->sigma_pop = res.sigma_pop; out->int_grad = res.int_grad; out->K = res.K; out->res = res.res;
    out->d0 = res.d0; out->u_max = res.u_max; out->u_rms = res.u_rms; out->un_max = res.un_max;
    out->ut_max = res.ut_max; out->massa_R = res.massa_R; out->massa_B = res.massa_B;
    out->qx = res.qx; out->qy = res.qy; out->min_f = res.min_f; out->SFx = res.SFx; out->SFy = res.SFy;
    out->neg_total = res.neg_total; out->neg_cor = res.neg_cor; out->n_ruim = res.n_ruim;
    out->n_ajuste = res.n_ajuste;
    return ok ? 1 : 0;
}

// mede_inclinada with gravar_perfil (Imm_INCL.cpp:404 at the last step): writes perfil.dat of the
// post-collision populations of the last step into directory `dir`.
int ref_incl_write_perfil(void *h, const char *dir) {
    RefIncl *r = (RefIncl *)h;
    LATTICE L = r->lattice;
    std::swap(L.inif_R, L.inif_R_new);
    std::swap(L.inif_B, L.inif_B_new);
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0) return 0;
    INCL res;
    mede_inclinada(r->geometry, L, r->p, r->q, res, r->forca, true);
    return chdir(cwd) == 0 ? 1 : 0;
}

void ref_incl_destroy(void *h) {
    RefIncl *r = (RefIncl *)h;
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
