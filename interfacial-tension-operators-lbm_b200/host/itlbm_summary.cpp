// itlbm_summary -- the analisar_lote.py table rows of finished case folders, from the command line.
//
//   itlbm_summary <csv> <root> <case-folder>...
//
// Appends one row per folder (drops and inclined strips told apart by inclinacao.txt) to <csv>, the
// same row itlbm_serve appends when a case retires; folders run by itlbm_ops / itlbm_incl or by the
// reference binaries can be tabulated this way without analisar_lote.py.  Exit code 1 when a folder
// has no finished resumo.dat.
#include <iostream>
#include <string>
#include <sys/stat.h>

#include "case_io.h"
#include "summary.h"

int main(int argc, char **argv) {
    if (argc < 4) {
        std::cerr << "usage: itlbm_summary <csv> <root> <case-folder>...\n";
        return 1;
    }
    int rc = 0;
    for (int a = 3; a < argc; a++) {
        const std::string dir = argv[a];
        struct stat st;
        const bool strip = stat(itlbm_host::join(dir, "inclinacao.txt").c_str(), &st) == 0;
        if (!itlbm_host::append_summary_row(argv[1], dir, argv[2], strip)) {
            std::cerr << "itlbm_summary: no finished resumo.dat in " << dir << "\n";
            rc = 1;
        }
    }
    return rc;
}
