#!/usr/bin/env python3
"""Extract golden vectors from the reference's shipped outputs into small committed fixtures.

Run once in a container that has the reference project:

    python tests/golden/make_golden.py --ref <reference project root>    (or set ITLBM_REFERENCE)

It writes
  lotes_subset.json   inputs and the first diagnostic rows (steps 0, 500, 1000) of a selection of the
                      stored runs under Lotes/ -- laplace.dat, iso.dat and galilean.dat of Imm_OPS
                      cases, inclinada.dat of Imm_INCL cases -- plus each case's resumo.dat line;
  e0_resultado.json   the numbers of E0_resultado.txt (the reference's analytic operator checks);
  analisar_e2.json    three stored Lotes/E2 folders (their resumo.dat and laplace.dat as text) with the
                      rows the reference's own analisar_lote.coleta makes of them (the only part of this
                      script that imports reference code: the batch-table rows of a Python reference).
Apart from analisar_lote.py nothing here runs the reference; the files are parsed as text.
"""
import argparse
import os
import json
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent

# (batch, case folder) pairs: every operator of E1 at R = 10 and 20, the translating drop of E4v at
# v0 = 0.25, one E2 point per operator and the E3 inclined strips at theta = 26.6 deg.
OPS = ["P1", "P3 chi=-0.4", "P3 chi=0.5", "P3 chi=2", "F1", "F2", "F3"]
CASES = ([("E1", f"{o}/R=10") for o in OPS] + [("E1", f"{o}/R=20") for o in OPS[:2] + OPS[4:5]] +
         [("E4v", f"{o}/v0=0.25") for o in OPS] +
         [("E2", f"{o}/tau=0.6/sigma=0.1") for o in OPS] +
         [("E3", f"{o}/pq=2,1") for o in OPS] + [("E3", "P3 chi=0.5/pq=1,1"), ("E3", "F2/pq=4,1")])


def read_data_in(path):
    """data_in.txt: alternating label / value tokens (LBM_functions.cpp:10-268)."""
    tok = path.read_text().split()
    vals = tok[0:1] + tok[2::2]
    names = ["geo", "Dim_Pixel", "steps", "files", "n_threads", "tau", "tau_nh", "rho", "tau_R",
             "tau_B", "tau_m", "rho_R", "rho_B", "fat_R_B", "fat_R_R", "fat_B_B", "recoll", "wett_R"]
    return dict(zip(names, vals))


def rows(path, n=3):
    out = []
    for line in path.read_text().splitlines():
        if line.startswith("#") or not line.strip():
            continue
        out.append(line.split())
        if len(out) >= n:
            break
    return out


def header(path):
    return path.read_text().splitlines()[0].lstrip("#").split()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ITLBM_REFERENCE"))
    a = ap.parse_args()
    if not a.ref:
        ap.error("give --ref <reference project root> or set ITLBM_REFERENCE")
    ref = Path(a.ref)
    cases = []
    for batch, folder in CASES:
        d = ref / "Lotes" / batch / folder
        if not d.exists():
            continue
        din = read_data_in(d / "data_in.txt")
        c = {
            "batch": batch, "folder": folder,
            "operador": (d / "operador.txt").read_text().strip(),
            "velocity": (d / "velocity.txt").read_text().strip() if (d / "velocity.txt").exists() else "0",
            "tau": float(din["tau_R"]), "fat_R_B": float(din["fat_R_B"]), "recoll": float(din["recoll"]),
            "rho_R": float(din["rho_R"]), "rho_B": float(din["rho_B"]), "steps": int(din["steps"]),
            "resumo_header": header(d / "resumo.dat"), "resumo": rows(d / "resumo.dat", 1)[0],
        }
        if (d / "inclinacao.txt").exists():
            c["program"] = "Imm_INCL"
            c["pq"] = [int(v) for v in (d / "inclinacao.txt").read_text().split()]
            c["N"] = int(c["resumo"][c["resumo_header"].index("N")])
            c["inclinada"] = rows(d / "inclinada.dat", 2)
        else:
            c["program"] = "Imm_OPS"
            c["nx"] = int(c["resumo"][c["resumo_header"].index("nx")])
            c["laplace"] = rows(d / "laplace.dat", 3)
            c["iso"] = rows(d / "iso.dat", 3)
            c["galilean"] = rows(d / "galilean.dat", 3)
            c["galilean_header"] = header(d / "galilean.dat")
        cases.append(c)
    (HERE / "lotes_subset.json").write_text(json.dumps(cases, indent=1))

    # E0_resultado.txt: "erro = <value>   ok" lines and the M4 table
    e0 = {"checks": [], "m4": {}}
    section = ""
    for line in (ref / "E0_resultado.txt").read_text().splitlines():
        m = re.match(r"\s*(.*?)\s+erro =\s*(\S+)\s+(ok|FALHOU)", line)
        if m:
            e0["checks"].append({"section": section, "what": m.group(1).strip(), "erro": float(m.group(2)),
                                 "status": m.group(3)})
            continue
        m4 = re.match(r"\s+(P1|P3 chi=\S+ \(\w+\))\s+((?:-?\d+\.\d+\s*){5})$", line)
        if m4 and "erro" not in line:
            e0["m4"][m4.group(1)] = [float(v) for v in m4.group(2).split()]
            continue
        if line.strip():
            section = line.strip()
    (HERE / "e0_resultado.json").write_text(json.dumps(e0, indent=1))
    # analisar_lote.coleta on stored E2 folders: three folders of different operators
    import importlib.util
    spec = importlib.util.spec_from_file_location("analisar_lote", ref / "analisar_lote.py")
    al = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(al)
    lotes = ref / "Lotes"
    picked, seen = [], set()
    for row in al.coleta(lotes, "E2"):
        op = row["pasta"].split("/")[0]
        if op in seen or op not in ("P3 chi=0.5", "F2", "P1"):
            continue
        seen.add(op)
        d = lotes / "E2" / row["pasta"]
        picked.append({"pasta": row["pasta"], "row": {k: (None if isinstance(v, float) and v != v else v)
                                                      for k, v in row.items()},
                       "resumo.dat": (d / "resumo.dat").read_text(), "laplace.dat": (d / "laplace.dat").read_text()})
    (HERE / "analisar_e2.json").write_text(json.dumps(picked, indent=1))
    print(f"{len(cases)} cases, {len(e0['checks'])} E0 checks, {len(e0['m4'])} M4 rows, "
          f"{len(picked)} analisar_lote rows")


if __name__ == "__main__":
    main()
