// case_io.cpp -- case-folder inputs and outputs (see case_io.h).
#include <cctype>
#include "case_io.h"

#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>

namespace itlbm_host {

std::string join(const std::string &dir, const std::string &file) {
    if (dir.empty() || dir == ".") return file;
    return dir.back() == '/' ? dir + file : dir + "/" + file;
}

// read_data (LBM_functions.cpp:10-268): the same token order and the same echo to stdout and
// dat_out.txt.
bool read_data(const std::string &dir, DataIn &d, std::ostream &log) {
    std::ifstream in(join(dir, "data_in.txt"));
    if (!in) {
        log << "\ndata_in.txt ausente." << std::endl;
        return false;
    }
    std::ofstream fdat(join(dir, "dat_out.txt"));
    auto both = [&](const std::string &first_cout, const std::string &first_fdat, auto &&... rest) {
        log << first_cout;
        fdat << first_fdat;
        ((log << rest), ...);
        ((fdat << rest), ...);
        log << std::endl;
        fdat << std::endl;
    };
    std::string label;
    log << "\nName of the output file: dat_out.txt" << std::endl;
    fdat << "Name of the output file: dat_out.txt" << std::endl;
    in >> d.geo_file;
    both("\nName of the geometry file: ", "\nName of the geometry file: ", d.geo_file);
    in >> label >> d.ftesc;
    both("\nPixel dimension = ", "\nPixel dimension = ", d.ftesc, " m");
    in >> label >> d.n_steps;
    both("\nNumber of steps: ", "\nNumber of steps: ", d.n_steps);
    in >> label >> d.n_files;
    both("\nNumber of files: ", "\nNumber of files: ", d.n_files);
    in >> label >> d.n_threads;
    both("\nNumber of threads: ", "\nNumber of threads: ", d.n_threads);
    in >> label >> d.tau;
    const double visc = (1. / 3.) * (d.tau - 0.5);
    both("\nRelaxation time: ", "\nRelaxation time: ", d.tau);
    both("\nKinematic viscosity = ", "\nKinematic viscosity = ", visc);
    in >> label >> d.tau_nh;
    both("\nRelaxation time (non-hidrodynamic): ", "\nRelaxation time (non-hidrodynamic): ", d.tau_nh);
    in >> label >> d.rho_ini;
    both("\nDensity: ", "\nDensity: ", d.rho_ini);
    in >> label >> d.tau_R;
    const double visc_R = (1.0 / 3.0) * (d.tau_R - 0.5);
    if (d.tau_R) both("\nRelaxation time (Red): ", "\nRelaxation time (Red): ", d.tau_R, " => viscosity R = ", visc_R);
    in >> label >> d.tau_B;
    const double visc_B = (1.0 / 3.0) * (d.tau_B - 0.5);
    if (d.tau_B) both("\nRelaxation time (Blue): ", "\nRelaxation time (Blue): ", d.tau_B, " => viscosity B = ", visc_B);
    in >> label >> d.tau_m;
    if (d.tau_R) both("\nRelaxation time (mixture): ", "\nRelaxation time (mixture): ", d.tau_m);
    in >> label >> d.rho_ini_R;
    if (d.tau_R) both("\nInitial density (Red): ", "\nInitial density (Red): ", d.rho_ini_R);
    in >> label >> d.rho_ini_B;
    if (d.tau_B) both("\nInitial density (Blue): ", "\nInitial density (Blue): ", d.rho_ini_B);
    in >> label >> d.A_fact;
    if (d.tau_R) both("\nInterfacial factor[0;0.4]: ", "\nInterfacial factor[0;0.4]: ", d.A_fact);
    in >> label >> d.A_fact_R;
    if (d.tau_R) both("\nInteraction factor (Red) [0;0.4]: ", "\nInteraction factor (Red) [0;0.4]: ", d.A_fact_R);
    in >> label >> d.A_fact_B;
    if (d.tau_B) both("\nInteraction factor (Blue) [0;0.4]: ", "\nInteraction factor (Blue) [0;0.4]: ", d.A_fact_B);
    in >> label >> d.recoll;
    if (d.tau_R) both("\nRecolloring factor[0;1]: ", "\nRecolloring factor[0;1]: ", d.recoll);
    in >> label >> d.wett_R;
    if (d.tau_R) both("\nRed_wall interaction [0.0 ; 1.0] : ", "\nRed_wall interaction [0.0 ; 1.0] : ", d.wett_R);
    return true;
}

// read_geo (LBM_functions.cpp:280-354) with pts_in = pts_out = 0
bool read_geometry(const std::string &path, int &nx, int &ny, int &nz, long long &n_fluid) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line, dump;
    for (int i = 0; i < 4; i++) std::getline(f, dump);
    std::getline(f, line);
    std::stringstream ss(line);
    nx = ny = nz = 0;
    ss >> dump >> nx >> ny >> nz;
    if (nx <= 0 || ny <= 0 || nz <= 0) return false;
    for (int i = 0; i < 5; i++) std::getline(f, dump);
    n_fluid = 0;
    const long long n = (long long)nx * ny * nz;
    for (long long k = 0; k < n; k++) {
        int v = 0;
        if (!(f >> v)) break;
        if (v) n_fluid++;
    }
    return true;
}

bool read_velocity(const std::string &dir, double &v0) {
    v0 = 0.0;
    std::ifstream vin(join(dir, "velocity.txt"));
    if (vin && !(vin >> v0)) v0 = 0.0;
    return std::isfinite(v0) && v0 >= 0.0;
}

bool read_inclinacao(const std::string &dir, int &p, int &q) {
    p = 1;
    q = 0;
    std::ifstream in(join(dir, "inclinacao.txt"));
    return (in >> p >> q) && !(p == 0 && q == 0);
}

void read_gota(const std::string &dir, double &radius, double &espessura) {
    radius = 0.0;
    espessura = 3.45;
    std::ifstream in(join(dir, "gota.txt"));
    if (!in) return;
    double r, e;
    if (in >> r) radius = r;
    if (in >> e) espessura = e;
}

void gi_header(std::ostream &out) {
    out << "# step v0 Mach sigma R umax_ref urms_ref umax_mean urms_mean umax_lab mean_x mean_y mean_z "
           "drop_ux drop_uy x0 y0 x_unwrapped center_dx center_dy axis_ratio mass_R mass_B min_f "
           "negative_total negative_color min_rho min_phi max_phi qx qy qz p_in p_out delta_p urms_lab\n";
}

void gi_write(std::ostream &out, int step, double v0, double cs2, const itlbm_drop_diag &d) {
    out << std::setprecision(17) << step << ' ' << v0 << ' ' << v0 / std::sqrt(cs2) << ' ' << d.sigma << ' '
        << d.raio << ' ' << d.max_ref << ' ' << d.rms_ref << ' ' << d.max_mean << ' ' << d.rms_mean << ' '
        << d.max_lab << ' ' << d.mean_x << ' ' << d.mean_y << ' ' << d.mean_z << ' ' << d.drop_x << ' '
        << d.drop_y << ' ' << d.x0 << ' ' << d.y0 << ' ' << d.x_unwrapped << ' ' << d.center_dx << ' '
        << d.center_dy << ' ' << d.axis_ratio << ' ' << d.massa_R << ' ' << d.massa_B << ' ' << d.min_f << ' '
        << d.negative_total << ' ' << d.negative_color << ' ' << d.min_rho << ' ' << d.min_phi << ' '
        << d.max_phi << ' ' << d.qx << ' ' << d.qy << ' ' << d.qz << ' ' << d.p_in << ' ' << d.p_out << ' '
        << d.delta_p << ' ' << d.rms_lab << '\n';
    out.flush();
}

bool write_vtk_scalar(const std::string &path, const char *title, const char *name, int nx, int ny,
                      const double *v) {
    std::ofstream f(path);
    if (!f) return false;
    f << "# vtk DataFile Version 2.0" << std::endl << title << std::endl << "ASCII" << std::endl
      << "DATASET STRUCTURED_POINTS" << std::endl << "DIMENSIONS " << nx << " " << ny << " " << 1 << std::endl
      << "ASPECT_RATIO 1 1 1" << std::endl << "ORIGIN 0 0 0" << std::endl << "POINT_DATA " << nx * ny
      << std::endl << "SCALARS " << name << " double" << std::endl << "LOOKUP_TABLE default" << std::endl;
    for (int y = 0; y < ny; y++) {
        for (int x = 0; x < nx; x++) f << v[(size_t)y * nx + x] << " ";
        f << std::endl;
    }
    return true;
}

bool write_vtk_velocity(const std::string &path, int nx, int ny, const double *ux, const double *uy,
                        const double *uz) {
    std::ofstream f(path);
    if (!f) return false;
    f << "# vtk DataFile Version 2.0" << std::endl << "Velocidade" << std::endl << "ASCII" << std::endl
      << "DATASET STRUCTURED_POINTS" << std::endl << "DIMENSIONS " << nx << " " << ny << " " << 1 << std::endl
      << "ASPECT_RATIO 1 1 1" << std::endl << "ORIGIN 0 0 0" << std::endl << "POINT_DATA " << nx * ny
      << std::endl << "VECTORS velocidade double" << std::endl;
    for (int y = 0; y < ny; y++) {
        for (int x = 0; x < nx; x++) {
            const size_t p = (size_t)y * nx + x;
            f << ux[p] << " " << uy[p] << " " << uz[p] << " ";
        }
        f << std::endl;
    }
    return true;
}

double dist_central(int x, int y, int p, int q, int N) {
    const double m = std::sqrt((double)(p * p + q * q));
    long long s = ((long long)p * x + (long long)q * y) % N;
    if (s < 0) s += N;
    double d = ((double)s - 0.5 * N);
    if (d >= 0.5 * N) d -= N;
    if (d < -0.5 * N) d += N;
    return -d / m;
}

bool write_perfil(const std::string &path, int N, int p, int q, const std::vector<double> &rR,
                  const std::vector<double> &rB, const std::vector<double> &ux,
                  const std::vector<double> &uy) {
    std::ofstream fp(path);
    if (!fp) return false;
    fp << "# d  c=rho_R/rho  rho  ux  uy\n" << std::setprecision(10);
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++) {
            const size_t k = (size_t)y * N + x;
            const double rho = rR[k] + rB[k];
            if (!(rho > 0)) continue;
            const double dd = dist_central(x, y, p, q, N);
            if (std::fabs(dd) < 12.0) fp << dd << " " << rR[k] / rho << " " << rho << " " << ux[k] << " " << uy[k] << "\n";
        }
    return true;
}

int precision_word(const char *word, int dflt) {
    if (!word) return dflt;
    std::string w(word);
    for (char &ch : w) ch = (char)std::tolower((unsigned char)ch);
    if (w == "fp64") return ITLBM_PREC_F64;
    if (w == "fp32") return ITLBM_PREC_F32;
    if (w == "fold") return ITLBM_PREC_F32_FOLD;
    return dflt;
}

const char *precision_label(int prec) {
    switch (prec) {
        case ITLBM_PREC_F32: return "FP32 ( f - w rho0 , f_R - f_B )";
        case ITLBM_PREC_F32_FOLD: return "FP32, nove classes no plano ( f - w rho0 , f_R - f_B )";
        default: return "FP64";
    }
}

}  // namespace itlbm_host
