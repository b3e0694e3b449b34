// itlbm_ops -- drop-in for the reference's Imm_OPS (static or translating cylindrical drop).
//
// Run with the case folder as the working directory (or give it as the only argument), exactly as
// rodar_lote.py runs Imm_OPS (rodar_lote.py:231-243).  Reads data_in.txt, operador.txt, velocity.txt
// and the geometry file; writes dat_out.txt, laplace.dat, iso.dat, galilean.dat, resumo.dat and the
// final VTK fields with the reference's layouts (Imm_OPS.cpp:65-404).  Exit code 1 on invalid input,
// 0 otherwise -- also when the run becomes unstable (estado = instavel in resumo.dat).
//
// Extensions (absent files keep the reference's behaviour): gota.txt "R [espessura]" sets the initial
// radius and the 10-90 % width of the initial profile (0 = sharp step); ITLBM_PRECISION=fp32 selects
// the FP32 shifted storage and =fold its nine-class in-plane fold; ITLBM_DEVICE selects the CUDA device.
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
const int PASSOS_DIAG = 500;      // Imm_OPS.cpp:44

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
    double v0 = 0.0;
    if (!read_velocity(dir, v0)) {
        std::cerr << "velocity.txt invalido.\n";
        return 1;
    }
    if (std::fabs(din.tau_R - din.tau_B) > 1e-14) {
        std::cerr << "\nEste programa usa BGK de tempo UNICO: tau_R e tau_B tem de ser iguais.\n";
        return 1;
    }
    int nx, ny, nz;
    long long n_fluid;
    if (!read_geometry(join(dir, din.geo_file), nx, ny, nz, n_fluid)) {
        std::cout << "\nNao foi possivel abrir " << din.geo_file << std::endl;
        return 1;
    }
    if (nz != 1 || n_fluid != (long long)nx * ny) {
        std::cerr << "\nEste programa requer caixa 2D periodica toda fluida ( nz = 1 ).\n";
        return 1;
    }
    double R_gota, espessura;
    read_gota(dir, R_gota, espessura);
    const double raio_ini = (R_gota > 0.0) ? R_gota : 0.25 * (double)nx;
    const int x0_ini = nx / 2, y0_ini = ny / 2;
    const bool forca = op.tipo >= ITLBM_OP_F1;
    const double tau = din.tau_R;
    const double A_in = din.A_fact;
    const double sigma_nominal = forca ? A_in : 4.0 / 9.0 * A_in * tau;
    const int prec = precision_word(std::getenv("ITLBM_PRECISION"), ITLBM_PREC_F64);
    if (const char *dev = std::getenv("ITLBM_DEVICE")) cudaSetDevice(std::atoi(dev));

    std::cout << "\nOperadores de tensao interfacial -- arcabouco comum ( D3Q19, BGK, Latva-Kokko )" << std::endl;
    std::cout << "   operador          = " << op.nome;
    if (op.tipo == ITLBM_OP_P3) std::cout << "   chi = " << op.chi;
    if (op.tipo == ITLBM_OP_F3) std::cout << "   xi = " << op.xi;
    std::cout << std::endl;
    std::cout << "   caixa             = " << nx << " x " << ny << " x " << nz << std::endl;
    std::cout << "   raio inicial      = " << raio_ini << std::endl;
    std::cout << "   tau               = " << tau << "   ( nu = " << (tau - 0.5) / 3.0 << " )" << std::endl;
    std::cout << "   beta              = " << din.recoll << std::endl;
    std::cout << "   fat_R_B           = " << A_in << (forca ? "   ( = sigma )" : "   ( = A )") << std::endl;
    std::cout << "   sigma nominal     = " << sigma_nominal << std::endl;
    std::cout << "   v0                = " << v0 << std::endl;
    std::cout << "   precisao          = " << precision_label(prec) << std::endl;

    itlbm_case_desc d{};
    d.nx = nx;
    d.ny = ny;
    d.op = op;
    d.tau = tau;
    d.beta = din.recoll;
    d.A_fact = A_in;
    d.rho_R = din.rho_ini_R;
    d.rho_B = din.rho_ini_B;
    d.geometry = ITLBM_GEOM_DROP;
    d.radius = raio_ini;
    d.k_profile = (espessura > 0.0) ? 2.0 * std::log(9.0) / espessura : 0.0;
    d.v0 = v0;
    d.precision = prec;
    itlbm_case *c = nullptr;
    if (itlbm_case_create(&d, &c) != ITLBM_OK) return die(c, 1, "itlbm_case_create");

    DropRun run;
    if (!run.open(dir, tau, v0, din.n_steps)) return die(c, 1, "cannot write the output files");
    const int n_steps = din.n_steps, n_files = din.n_files;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<double> rR, rB, ux, uy, uz;

    auto is_diag = [&](int s) { return (s % PASSOS_DIAG == 0) || (s == n_steps - 1); };
    auto is_vtk = [&](int s) {
        return s == n_steps - 1 || (n_files > 0 && s % std::max(1, n_steps / n_files) == 0 && s > 0);
    };
    int step = 0;
    while (step < n_steps) {
        // advance to the next step that is measured or written: the loop body of Imm_OPS.cpp:246-372
        int target = step;
        while (target < n_steps - 1 && !is_diag(target) && !is_vtk(target)) target++;
        if (itlbm_case_step(c, target - step + 1, ITLBM_STEP_KEEP_AUX, nullptr) != ITLBM_OK)
            return die(c, 2, "itlbm_case_step");
        step = target;
        if (step / 100 != (step - 1) / 100 || step == 0) std::cout << "\rStep : " << step << std::flush;
        if (is_diag(step)) {
            itlbm_drop_diag dg;
            if (itlbm_case_diag_drop(c, step, x0_ini, y0_ini, &dg, nullptr) != ITLBM_OK)
                return die(c, 2, "itlbm_case_diag_drop");
            if (run.on_diag(step, dg, &std::cout)) break;
        }
        if (is_vtk(step)) {  // GRAVA_CAMPOS_FINAIS, Imm_OPS.cpp:357-364
            const size_t n = (size_t)nx * ny;
            rR.resize(n); rB.resize(n); ux.resize(n); uy.resize(n); uz.resize(n);
            if (itlbm_case_read_fields(c, rR.data(), rB.data(), ux.data(), uy.data(), uz.data(), nullptr) != ITLBM_OK)
                return die(c, 2, "itlbm_case_read_fields");
            const std::string s = std::to_string((unsigned)step);
            write_vtk_scalar(join(dir, "rho_R" + s + ".vtk"), "Densidade", "densidade", nx, ny, rR.data());
            write_vtk_scalar(join(dir, "rho_B" + s + ".vtk"), "Densidade", "densidade", nx, ny, rB.data());
            write_vtk_velocity(join(dir, "vel_" + s + ".vtk"), nx, ny, ux.data(), uy.data(), uz.data());
        }
        step++;
    }
    itlbm_case_sync(c);
    itlbm_case_destroy(c);

    // resumo.dat (Imm_OPS.cpp:376-394)
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double mlups = (elapsed > 0) ? (double)n_fluid * step / (elapsed * 1e6) : 0.0;
    run.write_resumo(dir, op, tau, din.recoll, A_in, nx, raio_ini, sigma_nominal, step, mlups);
    const double m_sigma = run.n_med ? run.s_sigma / run.n_med : NAN;
    const double m_umax = run.n_med ? run.s_umax / run.n_med : NAN;
    std::cout << "\n\n================ Resultado ================" << std::endl;
    std::cout << "   estado            = " << run.estado << std::endl;
    std::cout << "   sigma ( media )   = " << m_sigma << "   ( nominal " << sigma_nominal << " )" << std::endl;
    std::cout << "   |u|max ( media )  = " << m_umax << "   |u|max / sigma = " << m_umax / m_sigma << std::endl;
    std::cout << "   populacoes < 0    = " << run.neg_total_max << " ( total )  " << run.neg_cor_max << " ( cor )" << std::endl;
    std::cout << "   MLUPS             = " << mlups << std::endl;
    return 0;
}
