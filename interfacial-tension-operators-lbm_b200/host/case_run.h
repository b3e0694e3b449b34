// case_run.h -- output accounting of one case: the diagnostic rows, the second-half means, the stop
// rule and resumo.dat, shared by the drop-in programs and the batch server.
//   DropRun   Imm_OPS.cpp:206-239 (files), :308-352 (rows, means, stop rule), :376-394 (resumo.dat)
//   StripRun  Imm_INCL.cpp:338-350, :404-434, :446-460
#pragma once

#include <array>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "case_io.h"

namespace itlbm_host {

struct DropRun {
    std::ofstream lap, iso, gi;
    double nu = 0, v0 = 0;
    int n_steps = 0;
    double s_sigma = 0, s_umax = 0, s_urms = 0, s_a4 = 0, s_a8 = 0, s_K = 0;
    int n_med = 0;
    long long neg_total_max = 0, neg_cor_max = 0;
    double min_f_global = 1e30;
    std::string estado = "estavel";
    int passo_falha = -1;

    // per diagnostic row, at full precision: step, sigma, u_max, u_rms, a4, a8, K_perfil,
    // negative_total, negative_color, min_f (what the means and maxima of resumo.dat are made of)
    std::vector<std::array<double, 10>> hist;

    bool open(const std::string &dir, double tau, double v0_, int n_steps_);
    // One diagnostic step; returns true when the stop rule fires (Imm_OPS.cpp:346-352).
    bool on_diag(int step, const itlbm_drop_diag &dg, std::ostream *log);
    // Resuming from a snapshot: keep the rows of laplace.dat, iso.dat and galilean.dat up to step
    // `upto`, append after them, and rebuild the accounting from the saved history (`hist_file`),
    // replayed in order so that the means come out as they would have without the interruption.
    bool resume(const std::string &dir, double tau, double v0_, int n_steps_, int upto,
                const std::string &hist_file);
    bool save_hist(const std::string &path) const;
    void account(const std::array<double, 10> &r);
    void write_resumo(const std::string &dir, const itlbm_operador &op, double tau, double beta,
                      double A_in, int nx, double raio_ini, double sigma_nominal, int steps,
                      double mlups) const;
};

struct StripRun {
    std::ofstream inc;
    int n_steps = 0, p = 1, q = 0;
    double s_sig = 0, s_um = 0, s_un = 0, s_ut = 0, s_K = 0, s_res = 0, s_ig = 0;
    int n_med = 0;
    long long neg_t = 0, neg_c = 0;
    double min_f = 1e300, d0_ini = NAN, d0_fim = NAN;
    std::string estado = "estavel";
    int passo_falha = -1;

    // per diagnostic row: step, sigma_pop, u_max, un_max, ut_max, K, res, int_grad, d0, neg_total,
    // neg_cor, min_f
    std::vector<std::array<double, 12>> hist;

    bool open(const std::string &dir, int n_steps_, int p_, int q_);
    bool on_diag(int step, const itlbm_strip_diag &r, std::ostream *log);
    bool resume(const std::string &dir, int n_steps_, int p_, int q_, int upto, const std::string &hist_file);
    bool save_hist(const std::string &path) const;
    void account(const std::array<double, 12> &r);
    void write_resumo(const std::string &dir, const itlbm_operador &op, double tau, double beta,
                      double A_in, int N, double theta, double sigma_nominal, int steps,
                      double mlups) const;
};

}  // namespace itlbm_host
