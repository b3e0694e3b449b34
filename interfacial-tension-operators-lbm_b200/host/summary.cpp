// summary.cpp -- see summary.h.
#include "summary.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <sys/stat.h>
#include <vector>

#include "case_io.h"

namespace itlbm_host {

namespace {

// num (analisar_lote.py:35-39): a float, or NaN when the text is not a number
double num(const std::string &s) {
    char *end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    return (end && *end == '\0' && !s.empty()) ? v : NAN;
}

std::vector<std::string> words(const std::string &line) {
    std::istringstream in(line);
    std::vector<std::string> w;
    for (std::string t; in >> t;) w.push_back(t);
    return w;
}

// media (analisar_lote.py:67-69): mean of the non-NaN values, NaN when there are none.  The sum is
// compensated (Neumaier's variant of Kahan summation), as Python's built-in sum() of floats is from
// Python 3.12 on, so that trends formed from near-equal means agree to the last bit.
double media(const std::vector<double> &xs) {
    double s = 0, c = 0;
    int n = 0;
    for (double x : xs)
        if (!std::isnan(x)) {
            const double t = s + x;
            c += (std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s;
            s = t;
            n++;
        }
    if (c != 0 && std::isfinite(c)) s += c;
    return n ? s / n : NAN;
}

std::string fmt(double v) {
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

std::string rel_path(const std::string &dir, const std::string &root) {
    if (!root.empty()) {
        const std::string r = root.back() == '/' ? root : root + "/";
        if (dir.compare(0, r.size(), r) == 0) return dir.substr(r.size());
    }
    return dir;
}

}  // namespace

bool append_summary_row(const std::string &csv, const std::string &case_dir, const std::string &root,
                        bool strip) {
    std::ifstream fr(join(case_dir, "resumo.dat"));
    std::string head, line;
    if (!fr || !std::getline(fr, head) || !std::getline(fr, line)) return false;
    if (!head.empty() && head[0] == '#') head = head.substr(1);
    // drops: the fixed column names of analisar_lote.py:28-30 (values missing from the line read as
    // NaN, :42-51); strips: the names of the resumo.dat header (:248-250)
    static const std::vector<std::string> cols_gota = {
        "operador", "chi", "xi", "tau", "beta", "fat_R_B", "v0", "nx", "R_ini", "sigma_nominal", "estado",
        "passo_falha", "passos", "sigma_med", "umax_med", "urms_med", "umax_sigma", "Ca_s", "a4_med", "a8_med",
        "K_med", "neg_total_max", "neg_cor_max", "min_f", "MLUPS", "umax_rel_media", "soma_Fx_med"};
    const std::vector<std::string> keys = strip ? words(head) : cols_gota, vals = words(line);
    if (vals.empty()) return false;
    const std::string pasta = rel_path(case_dir, root);
    const std::string rotulo = pasta.substr(0, pasta.find('/'));
    std::vector<std::string> cols = {"pasta", "rotulo"}, row = {pasta, rotulo};
    for (size_t k = 0; k < keys.size(); k++) {
        cols.push_back(keys[k]);
        const std::string v = k < vals.size() ? vals[k] : "nan";
        row.push_back((keys[k] == "operador" || keys[k] == "estado") ? v : fmt(num(v)));
    }
    if (!strip) {
        // coleta (analisar_lote.py:82-99): the trend of |u - v0|max (column 9 of laplace.dat) over the
        // last fifth against 50-70 %, and the means of sigma (column 8) and R (column 2) over the
        // second half of the rows
        std::vector<std::vector<double>> rows;
        std::ifstream fl(join(case_dir, "laplace.dat"));
        for (std::string ln; std::getline(fl, ln);) {
            if (ln.empty() || ln[0] == '#' || words(ln).empty()) continue;
            std::vector<double> r;
            for (const std::string &w : words(ln)) r.push_back(num(w));
            rows.push_back(r);
        }
        auto col = [&](size_t a, size_t b, size_t c) {
            std::vector<double> out;
            for (size_t k = a; k < b && k < rows.size(); k++) out.push_back(c < rows[k].size() ? rows[k][c] : NAN);
            return out;
        };
        const size_t n = rows.size();
        double tend = NAN;
        if (n >= 10) {  // tendencia (analisar_lote.py:72-79)
            const double fim = media(col((size_t)(0.8 * n), n, 8));
            const double meio = media(col((size_t)(0.5 * n), (size_t)(0.7 * n), 8));
            tend = meio > 0 ? fim / meio - 1.0 : NAN;
        }
        cols.insert(cols.end(), {"tendencia", "sigma_meiafinal", "R_meiafinal"});
        row.push_back(fmt(tend));
        row.push_back(fmt(n ? media(col(n / 2, n, 7)) : NAN));
        row.push_back(fmt(n ? media(col(n / 2, n, 1)) : NAN));
    }
    struct stat st;
    const bool fresh = stat(csv.c_str(), &st) != 0 || st.st_size == 0;
    std::ofstream out(csv, std::ios::app);
    if (!out) return false;
    auto put = [&](const std::vector<std::string> &v) {
        for (size_t k = 0; k < v.size(); k++) {
            const bool quote = v[k].find_first_of(",\"\n") != std::string::npos;
            if (k) out << ',';
            if (quote) {
                out << '"';
                for (char ch : v[k]) out << (ch == '"' ? "\"\"" : std::string(1, ch));
                out << '"';
            } else {
                out << v[k];
            }
        }
        out << "\r\n";  // csv.writer's line terminator
    };
    if (fresh) put(cols);
    put(row);
    return (bool)out;
}

}  // namespace itlbm_host
