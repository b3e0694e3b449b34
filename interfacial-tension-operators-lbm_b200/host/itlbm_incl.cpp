// itlbm_incl -- drop-in for the reference's Imm_INCL (straight interfaces inclined at atan(q/p)).
//
// Same file contract as Imm_INCL.cpp:192-473: reads data_in.txt, operador.txt, inclinacao.txt and the
// geometry file (an N x N x 1 all-fluid box); writes dat_out.txt, inclinada.dat every 500 steps and at
// the last step, perfil.dat at the last step and resumo.dat.  Exit code 1 on invalid input.
// ITLBM_PRECISION=fp32 selects the FP32 shifted storage; ITLBM_DEVICE selects the CUDA device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "case_io.h"

#include <cuda_runtime.h>

using namespace itlbm_host;

namespace {
const double ESPESSURA_INI = 3.45;  // Imm_INCL.cpp:41
const int PASSOS_DIAG = 500;        // Imm_INCL.cpp:42
const double U_LIMITE = 0.4;        // Imm_INCL.cpp:43
const double PI = 3.14159265358979323846;

// dist_central (Imm_INCL.cpp:74-83): signed distance to the central interface
double dist_central(int x, int y, int p, int q, int N) {
    const double m = std::sqrt((double)(p * p + q * q));
    long long s = ((long long)p * x + (long long)q * y) % N;
    if (s < 0) s += N;
    double d = ((double)s - 0.5 * N);
    if (d >= 0.5 * N) d -= N;
    if (d < -0.5 * N) d += N;
    return -d / m;
}

int die(itlbm_case *c, int rc, const char *what) {
    std::cerr << "\n" << what << ": " << itlbm_last_error() << std::endl;
    if (c) itlbm_case_destroy(c);
    return rc;
}
}  // namespace

int main(int argc, char **argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    DataIn din;
    if (!read_data(dir, din, std::cout)) return 1;
    itlbm_operador op;
    if (itlbm_operador_read(join(dir, "operador.txt").c_str(), &op) != ITLBM_OK) {
        std::cerr << "\noperador.txt ausente ou invalido.  Uma linha: P1 | P3 chi | F1 | F2 | F3 xi\n";
        return 1;
    }
    int p = 1, q = 0;
    if (!read_inclinacao(dir, p, q)) {
        std::cerr << "inclinacao.txt: \"p q\" inteiros, nao ambos nulos.\n";
        return 1;
    }
    if (std::fabs(din.tau_R - din.tau_B) > 1e-14) {
        std::cerr << "tau_R e tau_B tem de ser iguais.\n";
        return 1;
    }
    int nx, ny, nz;
    long long n_fluid;
    if (!read_geometry(join(dir, din.geo_file), nx, ny, nz, n_fluid)) {
        std::cout << "\nNao foi possivel abrir " << din.geo_file << std::endl;
        return 1;
    }
    const int N = nx;
    if (nz != 1 || ny != N || n_fluid != (long long)N * N) {
        std::cerr << "\nEste programa requer caixa quadrada N x N x 1, toda fluida.\n";
        return 1;
    }
    const double m = std::sqrt((double)(p * p + q * q));
    const double L = N / m;
    const double theta = std::atan2((double)q, (double)p) * 180.0 / PI;
    const double tau = din.tau_R;
    const double A_in = din.A_fact;
    const bool forca = op.tipo >= ITLBM_OP_F1;
    const double sigma_nominal = forca ? A_in : 4.0 / 9.0 * A_in * tau;
    const char *prec_env = std::getenv("ITLBM_PRECISION");
    const bool fp32 = prec_env && (std::strcmp(prec_env, "fp32") == 0 || std::strcmp(prec_env, "FP32") == 0);
    if (const char *dev = std::getenv("ITLBM_DEVICE")) cudaSetDevice(std::atoi(dev));

    std::cout << "\nInterface plana inclinada -- arcabouco comum ( D3Q19, BGK, Latva-Kokko )" << std::endl;
    std::cout << "   operador          = " << op.nome << std::endl;
    std::cout << "   caixa             = " << N << " x " << N << std::endl;
    std::cout << "   ( p , q )         = ( " << p << " , " << q << " )   theta = " << theta << " graus" << std::endl;
    std::cout << "   distancia entre interfaces = " << 0.5 * L << std::endl;
    std::cout << "   sigma nominal     = " << sigma_nominal << std::endl;
    if (0.5 * L < 8.0 * ESPESSURA_INI)
        std::cout << "   ATENCAO: interfaces a menos de 8 espessuras uma da outra; aumente N." << std::endl;

    itlbm_case_desc d{};
    d.nx = N;
    d.ny = N;
    d.op = op;
    d.tau = tau;
    d.beta = din.recoll;
    d.A_fact = A_in;
    d.rho_R = 1.0;
    d.rho_B = 1.0;
    d.geometry = ITLBM_GEOM_STRIP;
    d.p = p;
    d.q = q;
    d.precision = fp32 ? ITLBM_PREC_F32 : ITLBM_PREC_F64;
    itlbm_case *c = nullptr;
    if (itlbm_case_create(&d, &c) != ITLBM_OK) return die(c, 1, "itlbm_case_create");

    std::ofstream f_inc(join(dir, "inclinada.dat"));
    f_inc << std::setprecision(10);
    f_inc << "# 1:passo  2:sigma_pop  3:int_grad  4:K  5:espessura_10_90  6:residuo  7:d0  8:|u|max  9:|u|rms"
             "  10:|u_n|max  11:|u_t|max  12:massa_R  13:massa_B  14:qx  15:qy  16:soma_Fx  17:soma_Fy"
             "  18:min_f  19:neg_total  20:neg_cor\n";

    double s_sig = 0, s_um = 0, s_un = 0, s_ut = 0, s_K = 0, s_res = 0, s_ig = 0;
    int n_med = 0;
    long long neg_t = 0, neg_c = 0;
    double min_f = 1e300, d0_ini = NAN, d0_fim = NAN;
    std::string estado = "estavel";
    int passo_falha = -1;
    const int n_steps = din.n_steps;
    const auto t0 = std::chrono::steady_clock::now();
    int step = 0;
    while (step < n_steps) {
        int target = step;
        while (target < n_steps - 1 && target % PASSOS_DIAG != 0) target++;
        if (itlbm_case_step(c, target - step + 1, ITLBM_STEP_KEEP_AUX, nullptr) != ITLBM_OK)
            return die(c, 2, "itlbm_case_step");
        step = target;
        const bool ultimo = (step == n_steps - 1);
        if (step % PASSOS_DIAG == 0 || ultimo) {
            itlbm_strip_diag r;
            if (itlbm_case_diag_strip(c, step, &r, nullptr) != ITLBM_OK) return die(c, 2, "itlbm_case_diag_strip");
            const bool ok = r.ok != 0;
            if (ultimo) {  // perfil.dat, Imm_INCL.cpp:101, :162
                const size_t n = (size_t)N * N;
                std::vector<double> rR(n), rB(n), ux(n), uy(n);
                if (itlbm_case_read_fields(c, rR.data(), rB.data(), ux.data(), uy.data(), nullptr, nullptr) != ITLBM_OK)
                    return die(c, 2, "itlbm_case_read_fields");
                std::ofstream fp(join(dir, "perfil.dat"));
                fp << "# d  c=rho_R/rho  rho  ux  uy\n" << std::setprecision(10);
                for (int y = 0; y < N; y++)
                    for (int x = 0; x < N; x++) {
                        const size_t k = (size_t)y * N + x;
                        const double rho = rR[k] + rB[k];
                        if (!(rho > 0)) continue;
                        const double dd = dist_central(x, y, p, q, N);
                        if (std::fabs(dd) < 12.0)
                            fp << dd << " " << rR[k] / rho << " " << rho << " " << ux[k] << " " << uy[k] << "\n";
                    }
            }
            f_inc << step << " " << r.sigma_pop << " " << r.int_grad << " " << r.K << " "
                  << (r.K > 0 ? 2.0 * std::log(9.0) / r.K : 0.0) << " " << r.res << " " << r.d0 << " " << r.u_max
                  << " " << r.u_rms << " " << r.un_max << " " << r.ut_max << " " << r.massa_R << " " << r.massa_B
                  << " " << r.qx << " " << r.qy << " " << r.SFx << " " << r.SFy << " " << r.min_f << " "
                  << r.neg_total << " " << r.neg_cor << "\n";
            f_inc.flush();
            if (step == 0) d0_ini = r.d0;
            d0_fim = r.d0;
            neg_t = std::max(neg_t, r.neg_total);
            neg_c = std::max(neg_c, r.neg_cor);
            min_f = std::min(min_f, r.min_f);
            if (step >= n_steps / 2) {
                s_sig += r.sigma_pop;
                s_um += r.u_max;
                s_un += r.un_max;
                s_ut += r.ut_max;
                s_K += r.K;
                s_res += r.res;
                s_ig += r.int_grad;
                n_med++;
            }
            std::cout << "\rstep = " << step << "   sigma_pop = " << r.sigma_pop << "   K = " << r.K
                      << "   |u|max = " << r.u_max << "   neg = " << r.neg_total << "        " << std::endl;
            if (!ok || r.u_max > U_LIMITE) {
                estado = "instavel";
                passo_falha = step;
                std::cout << "\nSimulacao instavel no passo " << step << std::endl;
                break;
            }
        }
        step++;
    }
    itlbm_case_sync(c);
    itlbm_case_destroy(c);

    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double mlups = (elapsed > 0) ? (double)n_fluid * step / (elapsed * 1e6) : 0.0;
    auto med = [&](double s) { return n_med ? s / n_med : NAN; };
    std::ofstream f_res(join(dir, "resumo.dat"));
    f_res << std::setprecision(10);
    f_res << "# operador chi xi tau beta fat_R_B N p q theta sigma_nominal estado passo_falha passos "
             "sigma_pop_med int_grad_med K_med residuo_med umax_med un_max_med ut_max_med umax/sigma_nominal "
             "d0_ini d0_fim neg_total_max neg_cor_max min_f MLUPS\n";
    f_res << op.nome << " " << op.chi << " " << op.xi << " " << tau << " " << din.recoll << " " << A_in << " " << N
          << " " << p << " " << q << " " << theta << " " << sigma_nominal << " " << estado << " " << passo_falha << " "
          << step << " " << med(s_sig) << " " << med(s_ig) << " " << med(s_K) << " " << med(s_res) << " "
          << med(s_um) << " " << med(s_un) << " " << med(s_ut) << " " << med(s_um) / sigma_nominal << " " << d0_ini
          << " " << d0_fim << " " << neg_t << " " << neg_c << " " << min_f << " " << mlups << "\n";
    std::cout << "\n\n================ Resultado ================" << std::endl;
    std::cout << "   estado            = " << estado << std::endl;
    std::cout << "   theta             = " << theta << " graus" << std::endl;
    std::cout << "   sigma_pop         = " << med(s_sig) << "   ( nominal " << sigma_nominal << ";  ~0 nas forcas )" << std::endl;
    std::cout << "   int |grad|        = " << med(s_ig) << "   ( deve ser 2 )" << std::endl;
    std::cout << "   K / espessura     = " << med(s_K) << " / " << 2.0 * std::log(9.0) / med(s_K) << std::endl;
    std::cout << "   |u|max            = " << med(s_um) << "   ( |u_n| " << med(s_un) << ", |u_t| " << med(s_ut) << " )" << std::endl;
    std::cout << "   d0 inicial / final= " << d0_ini << " / " << d0_fim << std::endl;
    std::cout << "   MLUPS             = " << mlups << std::endl;
    return 0;
}
