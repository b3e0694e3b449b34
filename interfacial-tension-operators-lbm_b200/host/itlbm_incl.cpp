// itlbm_incl -- drop-in for the reference's Imm_INCL (straight interfaces inclined at atan(q/p)).
//
// Same file contract as Imm_INCL.cpp:192-473: reads data_in.txt, operador.txt, inclinacao.txt and the
// geometry file (an N x N x 1 all-fluid box); writes dat_out.txt, inclinada.dat every 500 steps and at
// the last step, perfil.dat at the last step and resumo.dat.  Exit code 1 on invalid input.
// ITLBM_PRECISION=fp32 selects the FP32 shifted storage and =fold its nine-class in-plane fold;
// ITLBM_DEVICE selects the CUDA device.
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
#include "case_run.h"

#include <cuda_runtime.h>

using namespace itlbm_host;

namespace {
const double ESPESSURA_INI = 3.45;  // Imm_INCL.cpp:41
const int PASSOS_DIAG = 500;        // Imm_INCL.cpp:42
const double PI = 3.14159265358979323846;

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
    const int prec = precision_word(std::getenv("ITLBM_PRECISION"), ITLBM_PREC_F64);
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
    d.precision = prec;
    itlbm_case *c = nullptr;
    if (itlbm_case_create(&d, &c) != ITLBM_OK) return die(c, 1, "itlbm_case_create");

    StripRun run;
    if (!run.open(dir, din.n_steps, p, q)) return die(c, 1, "cannot write the output files");
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
            if (ultimo) {  // perfil.dat, Imm_INCL.cpp:101, :162
                const size_t n = (size_t)N * N;
                std::vector<double> rR(n), rB(n), ux(n), uy(n);
                if (itlbm_case_read_profile(c, rR.data(), rB.data(), ux.data(), uy.data()) != ITLBM_OK)
                    return die(c, 2, "itlbm_case_read_profile");
                write_perfil(join(dir, "perfil.dat"), N, p, q, rR, rB, ux, uy);
            }
            if (run.on_diag(step, r, &std::cout)) break;
        }
        step++;
    }
    itlbm_case_sync(c);
    itlbm_case_destroy(c);

    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double mlups = (elapsed > 0) ? (double)n_fluid * step / (elapsed * 1e6) : 0.0;
    run.write_resumo(dir, op, tau, din.recoll, A_in, N, theta, sigma_nominal, step, mlups);
    auto med = [&](double s) { return run.n_med ? s / run.n_med : NAN; };
    const double s_sig = run.s_sig, s_ig = run.s_ig, s_K = run.s_K, s_um = run.s_um, s_un = run.s_un, s_ut = run.s_ut;
    const double d0_ini = run.d0_ini, d0_fim = run.d0_fim;
    const std::string &estado = run.estado;
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
