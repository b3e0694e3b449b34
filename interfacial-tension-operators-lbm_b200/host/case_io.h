// case_io.h -- the case-folder file contract of the reference programs, on the host.
//
// Inputs:  data_in.txt (read_data, SimBoltz_Functions/LBM_functions.cpp:10-268), operador.txt
//          (le_operador, Operadores_tensao.cpp:66-86), velocity.txt (Imm_OPS.cpp:82-87),
//          inclinacao.txt (Imm_INCL.cpp:208-212), the geometry file (read_geo, LBM_functions.cpp:280-354)
//          and, as an optional extension, gota.txt (drop radius and initial interface width).
// Outputs: dat_out.txt, laplace.dat, iso.dat, galilean.dat, resumo.dat, inclinada.dat, perfil.dat and
//          the final VTK fields, with the column layouts and precisions of the reference.
#pragma once

#include <cstdio>
#include <ostream>
#include <string>
#include <vector>

#include "../../include/itlbm.h"

namespace itlbm_host {

// data_in.txt: alternating label / value tokens in a fixed order; the labels are not checked.
struct DataIn {
    std::string geo_file;
    double ftesc = 0;
    int n_steps = 0, n_files = 0, n_threads = 0;
    double tau = 0, tau_nh = 0, rho_ini = 0, tau_R = 0, tau_B = 0, tau_m = 0;
    double rho_ini_R = 0, rho_ini_B = 0, A_fact = 0, A_fact_R = 0, A_fact_B = 0, recoll = 0, wett_R = 0;
};

// Reads data_in.txt from `dir` and writes dat_out.txt there; the echo also goes to `log`.
bool read_data(const std::string &dir, DataIn &d, std::ostream &log);

// Geometry header (DIMENSIONS line, 5th line) and body; counts fluid points (non-zero values).
bool read_geometry(const std::string &path, int &nx, int &ny, int &nz, long long &n_fluid);

// velocity.txt: absent -> 0, unreadable -> 0 (Imm_OPS.cpp:82-87).  Returns false when the value is
// not finite or negative.
bool read_velocity(const std::string &dir, double &v0);

// inclinacao.txt: "p q", integers, not both zero.
bool read_inclinacao(const std::string &dir, int &p, int &q);

// gota.txt (extension): "R [espessura]".  Absent -> R = nx / 4 and espessura 3.45 (Imm_OPS.cpp:39-40,
// 134, 199); espessura <= 0 selects a sharp initial step.
void read_gota(const std::string &dir, double &radius, double &espessura);

// gi_header / gi_write (Galilean_diagnostics.cpp:107-123)
void gi_header(std::ostream &out);
void gi_write(std::ostream &out, int step, double v0, double cs2, const itlbm_drop_diag &d);

// rec_density / rec_velocity (LBM_functions.cpp:1349-1511), from host fields in pto order.
bool write_vtk_scalar(const std::string &path, const char *title, const char *name, int nx, int ny,
                      const double *v);
bool write_vtk_velocity(const std::string &path, int nx, int ny, const double *ux, const double *uy,
                        const double *uz);

std::string join(const std::string &dir, const std::string &file);

// Storage form from an ITLBM_PRECISION word: "fp64", "fp32" or "fold" (either case); a null or other
// word gives `dflt`.  precision_label is the "precisao" line of the programs' banner.
int precision_word(const char *word, int dflt);
const char *precision_label(int prec);

// dist_central (Imm_INCL.cpp:74-83): signed distance to the central interface, > 0 on the red side
double dist_central(int x, int y, int p, int q, int N);

// perfil.dat (Imm_INCL.cpp:101, :162): d, c_R, rho, ux, uy of the nodes with |d| < 12, in y-major
// order, from the post-collision fields of the last step
bool write_perfil(const std::string &path, int N, int p, int q, const std::vector<double> &rR,
                  const std::vector<double> &rB, const std::vector<double> &ux,
                  const std::vector<double> &uy);

}  // namespace itlbm_host
