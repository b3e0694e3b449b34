// summary.h -- the batch tables of analisar_lote.py, kept up to date while the server runs.
//
// analisar_lote.py builds, after a batch has finished, one CSV row per case folder from its
// resumo.dat and laplace.dat (coleta, analisar_lote.py:82-99, for Imm_OPS folders; coleta_incl,
// :241-255, for Imm_INCL folders) and writes them with escreve_csv (:102-110).  The server appends the
// same row the moment a case retires, so the tables exist without a post-pass:
//   drops:  pasta, rotulo, the 27 resumo columns of analisar_lote.py, tendencia, sigma_meiafinal,
//           R_meiafinal
//   strips: pasta, rotulo, the resumo.dat columns (named by its header)
// `pasta` is the case folder relative to `root` (absolute when the folder is not under it) and
// `rotulo` its first component.
#pragma once

#include <string>

namespace itlbm_host {

// Appends the case folder's row to `csv` (writing the header first when the file is new or empty).
// Returns false when resumo.dat is missing or has no data line (the row is then skipped, as
// analisar_lote.py skips such folders) or the CSV cannot be written.
bool append_summary_row(const std::string &csv, const std::string &case_dir, const std::string &root,
                        bool strip);

}  // namespace itlbm_host
