// itlbm_serve -- continuous batching of case folders on one GPU.
//
//   itlbm_serve <spool-dir> [--budget-gb G] [--chunk K] [--fp64] [--idle-exit S] [--max-cases M]
//               [--summary-root DIR] [--snapshots]
//
// The reference runs one process per case folder (rodar_lote.py:231-243).  This server keeps one
// batch (itlbm_batch_*) on the device and admits case folders as they arrive:
//   * a request is a file <spool>/<name>.req whose first line is the path of a case folder (the
//     folder rodar_lote.monta writes: data_in.txt, operador.txt, velocity.txt, meio.vtk and, for the
//     inclined interface, inclinacao.txt); an optional second word "fp64", "fp32" or "fold" picks the storage;
//   * the server renames it <name>.run, validates the folder like Imm_OPS / Imm_INCL (an invalid folder
//     gets <name>.err with the message, the reference's exit code 1), and submits the case;
//   * requests that arrive while others run are admitted as memory and slots free up: every round is
//     one graph replay of all admitted cases, so their work overlaps on the device;
//   * diagnostic rows stream into the case folder as they fall due (laplace.dat, iso.dat, galilean.dat
//     or inclinada.dat, formats of the reference); at its last step or when the stop rule fires the
//     case retires, resumo.dat is written (rodar_lote.feito's completion test) and <name>.run becomes
//     <name>.done with its time-to-result;
//   * <spool>/serve_stats.json keeps the count, p50 / p99 time-to-result and the aggregate MLUPS;
//   * <spool>/resumo_gota.csv and resumo_incl.csv get each retired case's row of the batch tables of
//     analisar_lote.py (folders named relative to --summary-root), so they need no post-pass;
//   * with --snapshots, each case's state is saved in its folder (estado_itlbm.bin, with the
//     diagnostic history in estado_itlbm.run) at every diagnostic; a request for a folder holding a
//     snapshot of the same case short of its step count resumes from it instead of step 0 (the
//     reference restarts from step 0, rodar_lote.py:5-7), with the same results.
//   * a drop that finishes gets its final fields, rho_R<n>.vtk, rho_B<n>.vtk and vel_<n>.vtk at its
//     last step n (Imm_OPS.cpp:357-364; an unstable run stops before them), a strip that reaches its
//     last step gets perfil.dat (Imm_INCL.cpp:101, :162): the batch holds a retired case's state until
//     they are written;
// The client bin/itlbm_submit turns this into a drop-in for the Imm_OPS binary of rodar_lote.py.
// Fields at intermediate steps (data_in.txt `files` > 0; rodar_lote.py writes 0) are written by
// itlbm_ops only.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <vector>

#include "case_io.h"
#include "case_run.h"
#include "summary.h"

using namespace itlbm_host;

namespace {

struct Job {
    std::string name, dir;
    itlbm_case_desc desc{};
    bool strip = false;
    long long resume_steps = 0;  // > 0: restart from the folder's snapshot, taken after this many steps
    int n_steps = 0, nx = 0;
    double raio_ini = 0, sigma_nominal = 0, theta = 0, beta = 0, A = 0, tau = 0;
    double t_submit = 0;
    std::unique_ptr<DropRun> drop;
    std::unique_ptr<StripRun> stp;
};

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

std::vector<std::string> list_requests(const std::string &spool) {
    std::vector<std::string> out;
    DIR *d = opendir(spool.c_str());
    if (!d) return out;
    while (dirent *e = readdir(d)) {
        const std::string n = e->d_name;
        if (n.size() > 4 && n.compare(n.size() - 4, 4, ".req") == 0) out.push_back(n.substr(0, n.size() - 4));
    }
    closedir(d);
    std::sort(out.begin(), out.end());
    return out;
}

void write_text(const std::string &path, const std::string &text) {
    std::ofstream f(path + ".tmp");
    f << text;
    f.close();
    std::rename((path + ".tmp").c_str(), path.c_str());
}

const char *SNAP_FILE = "estado_itlbm.bin";  // the case's state after its last snapshot
const char *HIST_FILE = "estado_itlbm.run";  // its diagnostic history, for the resumo.dat means

bool same_desc(const itlbm_case_desc &a, const itlbm_case_desc &b) {
    return a.nx == b.nx && a.ny == b.ny && a.op.tipo == b.op.tipo && a.op.chi == b.op.chi && a.op.xi == b.op.xi &&
           a.tau == b.tau && a.beta == b.beta && a.A_fact == b.A_fact && a.rho_R == b.rho_R && a.rho_B == b.rho_B &&
           a.geometry == b.geometry && a.radius == b.radius && a.k_profile == b.k_profile && a.v0 == b.v0 &&
           a.p == b.p && a.q == b.q && a.precision == b.precision;
}

// Reads and validates a case folder like Imm_OPS.cpp:65-135 / Imm_INCL.cpp:192-266.  With
// `snapshots`, a folder holding a snapshot of the same case that is short of its step count resumes
// from it (its output files keep their rows up to the snapshot).
bool prepare(Job &j, int prec, bool snapshots, std::string &err) {
    std::ostringstream log;
    DataIn din;
    if (!read_data(j.dir, din, log)) {
        err = "data_in.txt ausente";
        return false;
    }
    itlbm_operador op;
    if (itlbm_operador_read(join(j.dir, "operador.txt").c_str(), &op) != ITLBM_OK) {
        err = "operador.txt ausente ou invalido.  Uma linha: P1 | P3 chi | F1 | F2 | F3 xi";
        return false;
    }
    int p = 1, q = 0;
    struct stat st;
    j.strip = stat(join(j.dir, "inclinacao.txt").c_str(), &st) == 0;
    double v0 = 0.0;
    if (j.strip) {
        if (!read_inclinacao(j.dir, p, q)) {
            err = "inclinacao.txt: \"p q\" inteiros, nao ambos nulos.";
            return false;
        }
    } else if (!read_velocity(j.dir, v0)) {
        err = "velocity.txt invalido.";
        return false;
    }
    if (std::fabs(din.tau_R - din.tau_B) > 1e-14) {
        err = "tau_R e tau_B tem de ser iguais.";
        return false;
    }
    int nx, ny, nz;
    long long n_fluid;
    if (!read_geometry(join(j.dir, din.geo_file), nx, ny, nz, n_fluid)) {
        err = "Nao foi possivel abrir " + din.geo_file;
        return false;
    }
    if (nz != 1 || n_fluid != (long long)nx * ny || (j.strip && nx != ny)) {
        err = j.strip ? "Este programa requer caixa quadrada N x N x 1, toda fluida."
                      : "Este programa requer caixa 2D periodica toda fluida ( nz = 1 ).";
        return false;
    }
    double R_gota, espessura;
    read_gota(j.dir, R_gota, espessura);
    itlbm_case_desc &d = j.desc;
    d.nx = nx;
    d.ny = ny;
    d.op = op;
    d.tau = din.tau_R;
    d.beta = din.recoll;
    d.A_fact = din.A_fact;
    d.rho_R = j.strip ? 1.0 : din.rho_ini_R;
    d.rho_B = j.strip ? 1.0 : din.rho_ini_B;
    d.geometry = j.strip ? ITLBM_GEOM_STRIP : ITLBM_GEOM_DROP;
    j.raio_ini = (R_gota > 0.0) ? R_gota : 0.25 * (double)nx;
    d.radius = j.raio_ini;
    d.k_profile = (espessura > 0.0) ? 2.0 * std::log(9.0) / espessura : 0.0;
    d.v0 = v0;
    d.p = p;
    d.q = q;
    d.precision = prec;
    j.n_steps = din.n_steps;
    j.nx = nx;
    j.tau = din.tau_R;
    j.beta = din.recoll;
    j.A = din.A_fact;
    j.sigma_nominal = op.tipo >= ITLBM_OP_F1 ? j.A : 4.0 / 9.0 * j.A * j.tau;
    j.theta = std::atan2((double)q, (double)p) * 180.0 / 3.14159265358979323846;
    if (j.n_steps < 1) {
        err = "steps < 1";
        return false;
    }
    j.resume_steps = 0;
    if (snapshots) {
        itlbm_case_desc sd;
        long long steps = 0;
        if (stat(join(j.dir, HIST_FILE).c_str(), &st) == 0 &&
            itlbm_snapshot_info(join(j.dir, SNAP_FILE).c_str(), &sd, &steps) == ITLBM_OK && same_desc(sd, d) &&
            steps > 0 && steps < j.n_steps)
            j.resume_steps = steps;
    }
    const int upto = (int)j.resume_steps - 1;  // the last diagnostic step before the snapshot
    if (j.strip) {
        j.stp.reset(new StripRun());
        const bool ok = j.resume_steps ? j.stp->resume(j.dir, j.n_steps, p, q, upto, join(j.dir, HIST_FILE))
                                       : j.stp->open(j.dir, j.n_steps, p, q);
        if (!ok) {
            err = "cannot write inclinada.dat";
            return false;
        }
    } else {
        j.drop.reset(new DropRun());
        const bool ok = j.resume_steps ? j.drop->resume(j.dir, j.tau, v0, j.n_steps, upto, join(j.dir, HIST_FILE))
                                       : j.drop->open(j.dir, j.tau, v0, j.n_steps);
        if (!ok) {
            err = "cannot write the output files";
            return false;
        }
    }
    return true;
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return NAN;
    std::sort(v.begin(), v.end());
    const double r = p * (v.size() - 1);
    const size_t i = (size_t)r;
    const double f = r - i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::cerr << "usage: itlbm_serve <spool-dir> [--budget-gb G] [--chunk K] [--fp64] [--idle-exit S] "
                     "[--max-cases M] [--summary-root DIR] [--snapshots]\n";
        return 1;
    }
    const std::string spool = argv[1];
    double budget_gb = 0, idle_exit = -1;
    int chunk = 500, max_cases = 0;
    bool fp64_default = false;
    std::string summary_root;  // case folders are named relative to it in the batch tables
    bool snapshots = false;    // snapshot every case at each diagnostic and resume from snapshots
    for (int a = 2; a < argc; a++) {
        const std::string k = argv[a];
        if (k == "--budget-gb" && a + 1 < argc) budget_gb = std::atof(argv[++a]);
        else if (k == "--chunk" && a + 1 < argc) chunk = std::atoi(argv[++a]);
        else if (k == "--idle-exit" && a + 1 < argc) idle_exit = std::atof(argv[++a]);
        else if (k == "--max-cases" && a + 1 < argc) max_cases = std::atoi(argv[++a]);
        else if (k == "--fp64") fp64_default = true;
        else if (k == "--summary-root" && a + 1 < argc) summary_root = argv[++a];
        else if (k == "--snapshots") snapshots = true;
    }
    itlbm_batch_config cfg{};
    cfg.hbm_budget = (size_t)(budget_gb * 1e9);
    cfg.chunk = chunk;
    cfg.diag_every = 500;
    cfg.max_cases = max_cases;
    itlbm_batch *b = nullptr;
    if (itlbm_batch_create(&cfg, &b) != ITLBM_OK) {
        std::cerr << "itlbm_batch_create: " << itlbm_last_error() << std::endl;
        return 2;
    }
    itlbm_batch_hold_finished(b, 1);  // retired cases wait for their final fields
    std::map<long long, Job> jobs;
    long long next_tag = 0;
    std::vector<double> latencies;
    const double t_start = now_s();
    double last_work = t_start;
    long long completed = 0, failed_inputs = 0;
    std::vector<itlbm_batch_event> ev(1024);
    while (true) {
        // new requests
        for (const std::string &name : list_requests(spool)) {
            const std::string req = join(spool, name + ".req"), run = join(spool, name + ".run");
            std::ifstream in(req);
            std::string dir, prec;
            in >> dir >> prec;
            in.close();
            if (std::rename(req.c_str(), run.c_str()) != 0) continue;
            Job j;
            j.name = name;
            j.dir = dir;
            std::string err;
            const int prec_code =
                precision_word(prec.c_str(), fp64_default ? ITLBM_PREC_F64 : ITLBM_PREC_F32);
            if (!prepare(j, prec_code, snapshots, err)) {
                write_text(join(spool, name + ".err"), err + "\n");
                std::remove(run.c_str());
                failed_inputs++;
                continue;
            }
            j.t_submit = now_s();
            const long long tag = next_tag++;
            const int sub = j.resume_steps
                                ? itlbm_batch_submit_saved(b, join(j.dir, SNAP_FILE).c_str(), j.n_steps, tag)
                                : itlbm_batch_submit(b, &j.desc, j.n_steps, tag);
            if (sub != ITLBM_OK) {
                write_text(join(spool, name + ".err"), std::string("admission: ") + itlbm_last_error() + "\n");
                std::remove(run.c_str());
                failed_inputs++;
                continue;
            }
            jobs.emplace(tag, std::move(j));
        }
        itlbm_batch_stats st;
        itlbm_batch_stats_get(b, &st);
        if (st.active == 0 && st.pending == 0) {
            if (idle_exit >= 0 && now_s() - last_work > idle_exit) break;
            std::this_thread::sleep_for(std::chrono::milliseconds(20));
            continue;
        }
        last_work = now_s();
        const int r = itlbm_batch_advance(b, nullptr);
        if (r < 0) {
            std::cerr << "itlbm_batch_advance: " << itlbm_last_error() << std::endl;
            break;
        }
        int n;
        while ((n = itlbm_batch_poll(b, ev.data(), (int)ev.size())) > 0) {
            for (int k = 0; k < n; k++) {
                const itlbm_batch_event &e = ev[k];
                auto it = jobs.find(e.tag);
                if (it == jobs.end()) continue;
                Job &j = it->second;
                if (e.kind == ITLBM_EV_DIAG) {
                    if (j.drop) j.drop->on_diag(e.step, e.drop, nullptr);
                    else j.stp->on_diag(e.step, e.strip, nullptr);
                    if (snapshots) {
                        // the history first, then the state (a case that retired in this round has no
                        // state left to save, and needs none)
                        const bool hist_ok = j.drop ? j.drop->save_hist(join(j.dir, HIST_FILE))
                                                    : j.stp->save_hist(join(j.dir, HIST_FILE));
                        const std::string snap = join(j.dir, SNAP_FILE);
                        const int rs = hist_ok ? itlbm_batch_save(b, e.tag, (snap + ".tmp").c_str()) : ITLBM_E_IO;
                        if (rs == ITLBM_OK) std::rename((snap + ".tmp").c_str(), snap.c_str());
                        else if (!(j.n_steps - 1 == e.step))  // the last step has no state left to save
                            std::cerr << "itlbm_serve: no snapshot of " << j.dir << " at step " << e.step << ": "
                                      << (hist_ok ? itlbm_last_error() : "history not written") << std::endl;
                    }
                    continue;
                }
                // final fields, read from the held state, then the case's memory goes back to the batch
                const int last = j.n_steps - 1;
                const size_t n = (size_t)j.desc.nx * j.desc.ny;
                if (j.drop && e.kind == ITLBM_EV_DONE) {
                    std::vector<double> rR(n), rB(n), ux(n), uy(n), uz(n);
                    if (itlbm_batch_read_fields(b, e.tag, ITLBM_FIELDS_VTK, rR.data(), rB.data(), ux.data(), uy.data(),
                                                uz.data()) == ITLBM_OK) {
                        const std::string sfx = std::to_string((unsigned)last);
                        write_vtk_scalar(join(j.dir, "rho_R" + sfx + ".vtk"), "Densidade", "densidade", j.desc.nx,
                                         j.desc.ny, rR.data());
                        write_vtk_scalar(join(j.dir, "rho_B" + sfx + ".vtk"), "Densidade", "densidade", j.desc.nx,
                                         j.desc.ny, rB.data());
                        write_vtk_velocity(join(j.dir, "vel_" + sfx + ".vtk"), j.desc.nx, j.desc.ny, ux.data(),
                                           uy.data(), uz.data());
                    } else {
                        std::cerr << "itlbm_serve: no final fields for " << j.dir << ": " << itlbm_last_error()
                                  << std::endl;
                    }
                } else if (!j.drop && (e.kind == ITLBM_EV_DONE || e.step == last)) {
                    std::vector<double> rR(n), rB(n), ux(n), uy(n);
                    if (itlbm_batch_read_fields(b, e.tag, ITLBM_FIELDS_PROFILE, rR.data(), rB.data(), ux.data(),
                                                uy.data(), nullptr) == ITLBM_OK)
                        write_perfil(join(j.dir, "perfil.dat"), j.desc.nx, j.desc.p, j.desc.q, rR, rB, ux, uy);
                    else
                        std::cerr << "itlbm_serve: no perfil.dat for " << j.dir << ": " << itlbm_last_error()
                                  << std::endl;
                }
                itlbm_batch_release(b, e.tag);
                const double t = now_s(), latency = t - j.t_submit;
                const int steps = e.step;
                const double mlups = latency > 0 ? (double)j.desc.nx * j.desc.ny * steps / (latency * 1e6) : 0;
                if (j.drop)
                    j.drop->write_resumo(j.dir, j.desc.op, j.tau, j.beta, j.A, j.nx, j.raio_ini, j.sigma_nominal,
                                         steps, mlups);
                else
                    j.stp->write_resumo(j.dir, j.desc.op, j.tau, j.beta, j.A, j.nx, j.theta, j.sigma_nominal,
                                        steps, mlups);
                // the analisar_lote.py tables, one row per retired case
                append_summary_row(join(spool, j.drop ? "resumo_gota.csv" : "resumo_incl.csv"), j.dir, summary_root,
                                   !j.drop);
                std::ostringstream done;
                done << std::setprecision(10) << (e.kind == ITLBM_EV_DONE ? "estavel" : "instavel") << " " << steps
                     << " " << latency << "\n";
                write_text(join(spool, j.name + ".done"), done.str());
                std::remove(join(spool, j.name + ".run").c_str());
                latencies.push_back(latency);
                completed++;
                jobs.erase(it);
            }
        }
        itlbm_batch_stats_get(b, &st);
        std::ostringstream js;
        const double wall = now_s() - t_start;
        js << std::setprecision(10) << "{\"completed\": " << completed << ", \"active\": " << st.active
           << ", \"pending\": " << st.pending << ", \"invalid\": " << failed_inputs
           << ", \"p50_s\": " << percentile(latencies, 0.5) << ", \"p99_s\": " << percentile(latencies, 0.99)
           << ", \"node_updates\": " << st.node_updates << ", \"device_ms\": " << st.device_ms
           << ", \"wall_s\": " << wall << ", \"mlups_wall\": " << st.node_updates / wall / 1e6
           << ", \"mlups_device\": " << (st.device_ms > 0 ? st.node_updates / (st.device_ms * 1e3) : 0.0)
           << ", \"diag_ms\": " << st.diag_ms << ", \"advance_ms\": " << st.advance_ms
           << ", \"admit_ms\": " << st.admit_ms << ", \"capture_ms\": " << st.capture_ms
           << ", \"captures\": " << st.captures << ", \"launch_mode\": " << st.launch_mode
           << ", \"hbm_used\": " << st.hbm_used << "}\n";
        std::string stats = js.str();
        for (size_t pos; (pos = stats.find("nan")) != std::string::npos;) stats.replace(pos, 3, "null");
        write_text(join(spool, "serve_stats.json"), stats);
    }
    itlbm_batch_destroy(b);
    return 0;
}
