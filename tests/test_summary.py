"""bin/itlbm_summary (and the server, which calls the same code as each case retires) writes the rows
of the batch tables of analisar_lote.py: for drop folders coleta (analisar_lote.py:82-99: the 27
resumo columns of :28-30, tendencia :72-79, sigma_meiafinal and R_meiafinal), for inclined-strip
folders coleta_incl (:241-255: the columns named by the resumo.dat header).  The expected rows are
restated here; where the reference's own analisar_lote.py is at hand it is also run on stored
folders of its batches and compared."""
import csv
import importlib.util
import os
import math
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
BIN = REPO / "interfacial-tension-operators-lbm_b200" / "bin" / "itlbm_summary"
# the reference project, where it is at hand ($ITLBM_REFERENCE): its own analisar_lote.py is then run too
REF = Path(os.environ.get("ITLBM_REFERENCE", "")) if os.environ.get("ITLBM_REFERENCE") else None

COLS = ['operador', 'chi', 'xi', 'tau', 'beta', 'fat_R_B', 'v0', 'nx', 'R_ini', 'sigma_nominal', 'estado',
        'passo_falha', 'passos', 'sigma_med', 'umax_med', 'urms_med', 'umax_sigma', 'Ca_s', 'a4_med', 'a8_med',
        'K_med', 'neg_total_max', 'neg_cor_max', 'min_f', 'MLUPS', 'umax_rel_media', 'soma_Fx_med']


def num(x):
    try:
        return float(x)
    except ValueError:
        return float("nan")


def media(xs):
    xs = [x for x in xs if not math.isnan(x)]
    return sum(xs) / len(xs) if xs else float("nan")


def expected_drop(d, root):
    lines = (d / "resumo.dat").read_text().strip().splitlines()
    row = dict(zip(COLS, lines[1].split()))
    for k in COLS:
        if k not in ("operador", "estado"):
            row[k] = num(row.get(k, "nan"))
    rows = [[num(x) for x in ln.split()] for ln in (d / "laplace.dat").read_text().splitlines()
            if ln.strip() and not ln.startswith("#")]
    n = len(rows)
    tend = float("nan")
    if n >= 10:
        fim = media([r[8] for r in rows[int(0.8 * n):]])
        meio = media([r[8] for r in rows[int(0.5 * n):int(0.7 * n)]])
        tend = fim / meio - 1.0 if meio > 0 else float("nan")
    pasta = str(d.relative_to(root))
    out = {"pasta": pasta, "rotulo": pasta.split("/")[0], **row, "tendencia": tend,
           "sigma_meiafinal": media([r[7] for r in rows[n // 2:]]) if rows else float("nan"),
           "R_meiafinal": media([r[1] for r in rows[n // 2:]]) if rows else float("nan")}
    return out


def same(a, b):
    if isinstance(a, float) or isinstance(b, float):
        fa, fb = num(str(a)), num(str(b))
        return (math.isnan(fa) and math.isnan(fb)) or fa == fb or abs(fa - fb) <= 1e-15 * abs(fa)
    return str(a) == str(b)


def write_drop(d, n_rows, estado="estavel", short=False):
    d.mkdir(parents=True)
    vals = ["P3", "0.5", "1.569988", "0.8", "0.8", "0.225", "0", "100", "25", "0.08", estado, "-1", "3001",
            "0.0812", "1.5e-05", "3e-06", "0.000185", "5.8e-05", "0.0012", "0.0003", "1.16", "0", "0", "0.0031",
            "12.5"]
    if short:
        vals = vals[:20]
    (d / "resumo.dat").write_text("# operador chi xi ... MLUPS\n" + " ".join(vals) + "\n")
    rows = ["# 1:passo ..."]
    for k in range(n_rows):
        r = [k * 500, 25 - 0.01 * k, 25.1, 25.2, 1.003, 0.999, 0.004, 0.08 + 1e-4 * k, 1e-5 * (1 + 0.1 * k),
             3e-6] + [0.1] * 12
        rows.append(" ".join(repr(x) for x in r))
    (d / "laplace.dat").write_text("\n".join(rows) + "\n")


def run(csv_path, root, *dirs):
    return subprocess.run([str(BIN), str(csv_path), str(root), *map(str, dirs)], capture_output=True, text=True)


def read_csv(p):
    with open(p, newline="") as f:
        return list(csv.DictReader(f))


def test_drop_rows_match_analisar_lote(tmp_path):
    root = tmp_path / "E2"
    cases = [root / "P3 chi=0.5" / "R=25" / "tau=0.8", root / "F2" / "R=10", root / "P1" / "curto"]
    write_drop(cases[0], 7)       # fewer than 10 rows: no trend
    write_drop(cases[1], 23, estado="instavel")
    write_drop(cases[2], 12, short=True)  # a resumo line with fewer columns
    out = tmp_path / "gota.csv"
    r = run(out, root, *cases)
    assert r.returncode == 0, r.stderr
    got = read_csv(out)
    assert list(got[0].keys()) == ["pasta", "rotulo"] + COLS + ["tendencia", "sigma_meiafinal", "R_meiafinal"]
    for d, g in zip(cases, got):
        e = expected_drop(d, root)
        for k, v in e.items():
            assert same(v, g[k]), (d.name, k, v, g[k])


def test_strip_rows_and_missing_folder(tmp_path):
    root = tmp_path / "E3"
    d = root / "F1" / "p=2 q=1"
    d.mkdir(parents=True)
    (d / "inclinacao.txt").write_text("2 1\n")
    (d / "resumo.dat").write_text("# operador chi xi tau N p q theta estado MLUPS\nF1 0.5 1.569988 1 200 2 1 "
                                  "26.56505118 estavel 9.5\n")
    empty = root / "P1" / "sem_resumo"
    empty.mkdir(parents=True)
    out = tmp_path / "incl.csv"
    r = run(out, root, d, empty)
    assert r.returncode == 1 and "sem_resumo" in r.stderr
    got = read_csv(out)
    assert len(got) == 1
    assert list(got[0].keys()) == ["pasta", "rotulo", "operador", "chi", "xi", "tau", "N", "p", "q", "theta",
                                   "estado", "MLUPS"]
    assert got[0]["pasta"] == "F1/p=2 q=1" and got[0]["rotulo"] == "F1" and float(got[0]["theta"]) == 26.56505118
    # appending keeps one header
    assert run(out, root, d).returncode == 0
    assert len(read_csv(out)) == 2


@pytest.mark.skipif(REF is None or not (REF / "analisar_lote.py").exists(),
                    reason="the reference is not at hand (set ITLBM_REFERENCE)")
def test_reference_tables_on_stored_folders(tmp_path):
    spec = importlib.util.spec_from_file_location("analisar_lote", REF / "analisar_lote.py")
    al = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(al)
    lotes = REF / "Lotes"
    ref_rows = al.coleta(lotes, "E2")[:12]
    assert ref_rows
    out = tmp_path / "e2.csv"
    dirs = [lotes / "E2" / r["pasta"] for r in ref_rows]
    assert run(out, lotes / "E2", *dirs).returncode == 0
    got = read_csv(out)
    for e, g in zip(ref_rows, got):
        for k, v in e.items():
            assert same(v, g[k]), (e["pasta"], k, v, g[k])


def test_stored_folders_match_analisar_lote_rows(tmp_path, golden):
    """Three stored Lotes/E2 folders (tests/golden/analisar_e2.json) and the rows the reference's own
    analisar_lote.coleta made of them: itlbm_summary writes the same rows."""
    import json
    fixture = json.loads((REPO / "tests" / "golden" / "analisar_e2.json").read_text())
    assert len(fixture) == 3
    root = tmp_path / "E2"
    dirs = []
    for f in fixture:
        d = root / f["pasta"]
        d.mkdir(parents=True)
        (d / "resumo.dat").write_text(f["resumo.dat"])
        (d / "laplace.dat").write_text(f["laplace.dat"])
        dirs.append(d)
    out = tmp_path / "e2.csv"
    assert run(out, root, *dirs).returncode == 0
    got = read_csv(out)
    for f, g in zip(fixture, got):
        for k, v in f["row"].items():
            assert same(float("nan") if v is None else v, g[k]), (f["pasta"], k, v, g[k])
