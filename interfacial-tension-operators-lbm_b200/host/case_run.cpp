// case_run.cpp -- see case_run.h.
#include "case_run.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>

namespace itlbm_host {

namespace {
const double U_LIMITE = 0.4;  // Imm_OPS.cpp:45, Imm_INCL.cpp:43
}

namespace {

// Rows of a diagnostic text file with a step number (first column) up to `upto`, header lines kept.
std::string rows_upto(const std::string &path, int upto) {
    std::ifstream in(path);
    std::string out, ln;
    while (std::getline(in, ln)) {
        if (!ln.empty() && ln[0] != '#') {
            std::istringstream ss(ln);
            double st;
            if (!(ss >> st) || st > upto) continue;
        }
        out += ln + "\n";
    }
    return out;
}

bool reopen(std::ofstream &f, const std::string &path, int upto) {
    const std::string kept = rows_upto(path, upto);
    f.open(path);
    if (!f) return false;
    f << kept;
    f.flush();
    return true;
}

template <size_t N>
bool write_hist(const std::string &path, const std::vector<std::array<double, N>> &h) {
    std::ofstream f(path + ".tmp");
    if (!f) return false;
    char b[40];
    for (const auto &r : h) {
        for (size_t k = 0; k < N; k++) {
            std::snprintf(b, sizeof b, "%a", r[k]);  // exact
            f << (k ? " " : "") << b;
        }
        f << "\n";
    }
    f.close();
    return std::rename((path + ".tmp").c_str(), path.c_str()) == 0;
}

template <size_t N>
bool read_hist(const std::string &path, int upto, std::vector<std::array<double, N>> &h) {
    std::ifstream f(path);
    if (!f) return false;
    h.clear();
    for (std::string ln; std::getline(f, ln);) {
        std::istringstream ss(ln);
        std::array<double, N> r{};
        std::string w;
        size_t k = 0;
        for (; k < N && ss >> w; k++) r[k] = std::strtod(w.c_str(), nullptr);
        if (k != N) return false;
        if (r[0] <= upto) h.push_back(r);
    }
    return true;
}

}  // namespace

void DropRun::account(const std::array<double, 10> &r) {
    const int step = (int)r[0];
    neg_total_max = std::max(neg_total_max, (long long)r[7]);
    neg_cor_max = std::max(neg_cor_max, (long long)r[8]);
    min_f_global = std::min(min_f_global, r[9]);
    if (step >= n_steps / 2) {
        s_sigma += r[1];
        s_umax += r[2];
        s_urms += r[3];
        s_a4 += r[4];
        s_a8 += r[5];
        s_K += r[6];
        n_med++;
    }
}

bool DropRun::save_hist(const std::string &path) const { return write_hist(path, hist); }

bool DropRun::resume(const std::string &dir, double tau, double v0_, int n_steps_, int upto,
                     const std::string &hist_file) {
    nu = (1. / 3.) * (tau - 0.5);
    v0 = v0_;
    n_steps = n_steps_;
    if (!read_hist(hist_file, upto, hist)) return false;
    for (const auto &r : hist) account(r);
    if (!(reopen(lap, join(dir, "laplace.dat"), upto) && reopen(iso, join(dir, "iso.dat"), upto) &&
          reopen(gi, join(dir, "galilean.dat"), upto)))
        return false;
    lap << std::setprecision(10);  // as open() sets them
    iso << std::setprecision(10);
    return true;
}

bool DropRun::open(const std::string &dir, double tau, double v0_, int n_steps_) {
    nu = (1. / 3.) * (tau - 0.5);
    v0 = v0_;
    n_steps = n_steps_;
    lap.open(join(dir, "laplace.dat"));
    iso.open(join(dir, "iso.dat"));
    gi.open(join(dir, "galilean.dat"));
    if (!lap || !iso || !gi) return false;
    lap << std::setprecision(10);
    lap << "# 1:passo  2:raio_area  3:raio_grad  4:raio_linha  5:p_in  6:p_out  7:delta_p"
           "  8:sigma  9:|u-v0|max  10:|u-v0|rms  11:Ca  12:massa_R  13:massa_B  14:|q|"
           "  15:sd_p_in  16:sd_p_out  17:sigma_2pontos"
           "  18:K_perfil  19:r_perfil  20:espessura_10_90  21:residuo_ajuste  22:n_camadas\n";
    iso << std::setprecision(10);
    iso << "# 1:passo  2:R0  3:|a2|/R0  4:|a4|/R0  5:|a8|/R0  6:rmin  7:rmax\n";
    gi_header(gi);
    return true;
}

bool DropRun::on_diag(int step, const itlbm_drop_diag &dg, std::ostream *log) {
    const bool ok = dg.ok != 0;
    if (ok) {
        const double Ca = (dg.sigma > 0.0) ? nu * dg.u_max / dg.sigma : 0.0;
        const double q = std::sqrt(dg.qx * dg.qx + dg.qy * dg.qy + dg.qz * dg.qz);
        lap << step << " " << dg.raio << " " << dg.raio_grad << " " << dg.raio_linha << " " << dg.p_in << " "
            << dg.p_out << " " << dg.delta_p << " " << dg.sigma << " " << dg.u_max << " " << dg.u_rms << " " << Ca
            << " " << dg.massa_R << " " << dg.massa_B << " " << q << " " << dg.sd_in << " " << dg.sd_out << " "
            << dg.sigma_linha << " " << dg.K_perfil << " " << dg.r_perfil << " " << dg.esp_perfil << " "
            << dg.res_perfil << " " << dg.n_perfil << "\n";
        lap.flush();
        gi_write(gi, step, v0, 1. / 3., dg);
        iso << step << " " << dg.R0 << " " << dg.a2 << " " << dg.a4 << " " << dg.a8 << " " << dg.rmin << " "
            << dg.rmax << "\n";
        iso.flush();
        hist.push_back({(double)step, dg.sigma, dg.u_max, dg.u_rms, dg.a4, dg.a8, dg.K_perfil,
                        (double)dg.negative_total, (double)dg.negative_color, dg.min_f});
        account(hist.back());
        if (log)
            *log << "\rstep = " << step << "   R = " << dg.raio << "   sigma = " << dg.sigma
                 << "   |u|max = " << dg.u_max << "   a4 = " << dg.a4 << "   neg = " << dg.negative_total
                 << "        " << std::endl;
    }
    if (!ok || dg.n_ruim > 0 || dg.u_max > U_LIMITE) {
        estado = "instavel";
        passo_falha = step;
        if (log) *log << "\nSimulacao instavel no passo " << step << std::endl;
        return true;
    }
    return false;
}

void DropRun::write_resumo(const std::string &dir, const itlbm_operador &op, double tau, double beta,
                           double A_in, int nx, double raio_ini, double sigma_nominal, int steps,
                           double mlups) const {
    const double m_sigma = n_med ? s_sigma / n_med : NAN;
    const double m_umax = n_med ? s_umax / n_med : NAN;
    std::ofstream f_res(join(dir, "resumo.dat"));
    f_res << std::setprecision(10);
    f_res << "# operador chi xi tau beta fat_R_B v0 nx R_ini sigma_nominal estado passo_falha passos "
             "sigma_med umax_med urms_med umax/sigma Ca_s=nu*umax/sigma a4_med a8_med K_med "
             "neg_total_max neg_cor_max min_f MLUPS\n";
    f_res << op.nome << " " << op.chi << " " << op.xi << " " << tau << " " << beta << " " << A_in << " " << v0
          << " " << nx << " " << raio_ini << " " << sigma_nominal << " " << estado << " " << passo_falha << " "
          << steps << " " << m_sigma << " " << m_umax << " " << (n_med ? s_urms / n_med : NAN) << " "
          << m_umax / m_sigma << " " << nu * m_umax / m_sigma << " " << (n_med ? s_a4 / n_med : NAN) << " "
          << (n_med ? s_a8 / n_med : NAN) << " " << (n_med ? s_K / n_med : NAN) << " " << neg_total_max << " "
          << neg_cor_max << " " << min_f_global << " " << mlups << "\n";
}

bool StripRun::open(const std::string &dir, int n_steps_, int p_, int q_) {
    n_steps = n_steps_;
    p = p_;
    q = q_;
    inc.open(join(dir, "inclinada.dat"));
    if (!inc) return false;
    inc << std::setprecision(10);
    inc << "# 1:passo  2:sigma_pop  3:int_grad  4:K  5:espessura_10_90  6:residuo  7:d0  8:|u|max  9:|u|rms"
           "  10:|u_n|max  11:|u_t|max  12:massa_R  13:massa_B  14:qx  15:qy  16:soma_Fx  17:soma_Fy"
           "  18:min_f  19:neg_total  20:neg_cor\n";
    return true;
}

void StripRun::account(const std::array<double, 12> &r) {
    const int step = (int)r[0];
    if (step == 0) d0_ini = r[8];
    d0_fim = r[8];
    neg_t = std::max(neg_t, (long long)r[9]);
    neg_c = std::max(neg_c, (long long)r[10]);
    min_f = std::min(min_f, r[11]);
    if (step >= n_steps / 2) {
        s_sig += r[1];
        s_um += r[2];
        s_un += r[3];
        s_ut += r[4];
        s_K += r[5];
        s_res += r[6];
        s_ig += r[7];
        n_med++;
    }
}

bool StripRun::save_hist(const std::string &path) const { return write_hist(path, hist); }

bool StripRun::resume(const std::string &dir, int n_steps_, int p_, int q_, int upto,
                      const std::string &hist_file) {
    n_steps = n_steps_;
    p = p_;
    q = q_;
    if (!read_hist(hist_file, upto, hist)) return false;
    for (const auto &r : hist) account(r);
    if (!reopen(inc, join(dir, "inclinada.dat"), upto)) return false;
    inc << std::setprecision(10);
    return true;
}

bool StripRun::on_diag(int step, const itlbm_strip_diag &r, std::ostream *log) {
    const bool ok = r.ok != 0;
    inc << step << " " << r.sigma_pop << " " << r.int_grad << " " << r.K << " "
        << (r.K > 0 ? 2.0 * std::log(9.0) / r.K : 0.0) << " " << r.res << " " << r.d0 << " " << r.u_max << " "
        << r.u_rms << " " << r.un_max << " " << r.ut_max << " " << r.massa_R << " " << r.massa_B << " " << r.qx
        << " " << r.qy << " " << r.SFx << " " << r.SFy << " " << r.min_f << " " << r.neg_total << " "
        << r.neg_cor << "\n";
    inc.flush();
    hist.push_back({(double)step, r.sigma_pop, r.u_max, r.un_max, r.ut_max, r.K, r.res, r.int_grad, r.d0,
                    (double)r.neg_total, (double)r.neg_cor, r.min_f});
    account(hist.back());
    if (log)
        *log << "\rstep = " << step << "   sigma_pop = " << r.sigma_pop << "   K = " << r.K
             << "   |u|max = " << r.u_max << "   neg = " << r.neg_total << "        " << std::endl;
    if (!ok || r.u_max > U_LIMITE) {
        estado = "instavel";
        passo_falha = step;
        if (log) *log << "\nSimulacao instavel no passo " << step << std::endl;
        return true;
    }
    return false;
}

void StripRun::write_resumo(const std::string &dir, const itlbm_operador &op, double tau, double beta,
                            double A_in, int N, double theta, double sigma_nominal, int steps,
                            double mlups) const {
    auto med = [&](double s) { return n_med ? s / n_med : NAN; };
    std::ofstream f_res(join(dir, "resumo.dat"));
    f_res << std::setprecision(10);
    f_res << "# operador chi xi tau beta fat_R_B N p q theta sigma_nominal estado passo_falha passos "
             "sigma_pop_med int_grad_med K_med residuo_med umax_med un_max_med ut_max_med umax/sigma_nominal "
             "d0_ini d0_fim neg_total_max neg_cor_max min_f MLUPS\n";
    f_res << op.nome << " " << op.chi << " " << op.xi << " " << tau << " " << beta << " " << A_in << " " << N << " "
          << p << " " << q << " " << theta << " " << sigma_nominal << " " << estado << " " << passo_falha << " "
          << steps << " " << med(s_sig) << " " << med(s_ig) << " " << med(s_K) << " " << med(s_res) << " "
          << med(s_um) << " " << med(s_un) << " " << med(s_ut) << " " << med(s_um) / sigma_nominal << " " << d0_ini
          << " " << d0_fim << " " << neg_t << " " << neg_c << " " << min_f << " " << mlups << "\n";
}

}  // namespace itlbm_host
