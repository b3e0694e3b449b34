// itlbm_submit -- client of itlbm_serve with the process contract of Imm_OPS / Imm_INCL.
//
// Run in a case folder (or with the folder as its argument), exactly like the reference binaries
// rodar_lote.py runs (rodar_lote.py:231-243).  It drops a request into the server's spool directory
// ($ITLBM_SPOOL), waits until the server has finished the case, and exits 0 when the case ran
// (stable or not, resumo.dat written by the server) or 1 when the folder was invalid (the message of
// the server on stderr).  ITLBM_PRECISION (fp64, fp32 or fold) picks the storage; ITLBM_SUBMIT_TIMEOUT
// bounds the wait in seconds (default: none).
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>

int main(int argc, char **argv) {
    const char *spool = std::getenv("ITLBM_SPOOL");
    if (!spool) {
        std::cerr << "itlbm_submit: set ITLBM_SPOOL to the spool directory of itlbm_serve\n";
        return 1;
    }
    char buf[PATH_MAX];
    std::string dir = argc > 1 ? argv[1] : ".";
    if (!realpath(dir.c_str(), buf)) {
        std::cerr << "itlbm_submit: no such folder " << dir << "\n";
        return 1;
    }
    dir = buf;
    const char *prec = std::getenv("ITLBM_PRECISION");
    std::ostringstream name;
    name << "req_" << getpid() << "_" << std::chrono::steady_clock::now().time_since_epoch().count();
    const std::string base = std::string(spool) + "/" + name.str();
    {
        std::ofstream f(base + ".tmp");
        f << dir << " " << (prec ? prec : "") << "\n";
    }
    std::rename((base + ".tmp").c_str(), (base + ".req").c_str());
    const char *to = std::getenv("ITLBM_SUBMIT_TIMEOUT");
    const double limit = to ? std::atof(to) : -1;
    const auto t0 = std::chrono::steady_clock::now();
    struct stat st;
    while (true) {
        if (stat((base + ".done").c_str(), &st) == 0) {
            std::ifstream f(base + ".done");
            std::string estado;
            int steps;
            double latency;
            f >> estado >> steps >> latency;
            std::cout << "estado = " << estado << "   passos = " << steps << "   tempo = " << latency << " s\n";
            std::remove((base + ".done").c_str());
            return 0;
        }
        if (stat((base + ".err").c_str(), &st) == 0) {
            std::ifstream f(base + ".err");
            std::cerr << f.rdbuf();
            std::remove((base + ".err").c_str());
            return 1;
        }
        const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (limit >= 0 && waited > limit) {
            std::cerr << "itlbm_submit: no answer from the server after " << waited << " s\n";
            return 2;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(50));
    }
}
