"""Serving: bin/itlbm_serve batches case folders that arrive while others run; bin/itlbm_submit gives
each request the process contract of Imm_OPS (the way rodar_lote.py runs it).  A case gives the same
result served in the mix as run alone: in FP64 the served diagnostic files are byte-identical to
those of bin/itlbm_ops on the same folder, the final fields (rho_R / rho_B / vel_ VTK files of a
drop, perfil.dat of a strip) included."""
import os
import subprocess
import threading
import time
from pathlib import Path

import pytest

from test_dropin import BIN, make_case, run

pytestmark = pytest.mark.gpu


def submit(d, spool, prec="fp64"):
    env = dict(os.environ, ITLBM_SPOOL=str(spool), ITLBM_PRECISION=prec, ITLBM_SUBMIT_TIMEOUT="300")
    return subprocess.run([str(BIN / "itlbm_submit")], cwd=d, capture_output=True, text=True, timeout=400, env=env)


def test_served_equals_alone_and_overlaps(tmp_path):
    spool = tmp_path / "spool"
    spool.mkdir()
    server = subprocess.Popen([str(BIN / "itlbm_serve"), str(spool), "--idle-exit", "3", "--chunk", "250",
                               "--summary-root", str(tmp_path)],
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        cases = [("P3 0.5", 0.225, 40, 1501, None), ("F2", 0.1, 56, 1200, None), ("F3 1.569988", 0.1, 48, 999, None),
                 ("P1", 0.225, 32, 2001, None), ("P3 2", 0.1, 40, 1001, (2, 1)), ("F1", 0.1, 36, 777, (1, 1))]
        dirs = [make_case(tmp_path / f"s{k}", op, A, 0.8, nx, steps, pq=pq) for k, (op, A, nx, steps, pq) in
                enumerate(cases)]
        results = [None] * len(dirs)

        def go(k, delay):
            time.sleep(delay)
            results[k] = submit(dirs[k], spool)

        threads = [threading.Thread(target=go, args=(k, 0.4 * k)) for k in range(len(dirs))]
        for t in threads:
            t.start()
        bad = make_case(tmp_path / "bad", "Z9", 0.1, 0.8, 32, 100)
        rbad = submit(bad, spool)
        for t in threads:
            t.join()
        assert rbad.returncode == 1 and "operador" in rbad.stderr
        for k, r in enumerate(results):
            assert r.returncode == 0, (k, r.stdout, r.stderr)
            assert "estado = estavel" in r.stdout
    finally:
        server.wait(timeout=120)
    # the same folders run alone by the drop-in programs
    for k, (op, A, nx, steps, pq) in enumerate(cases):
        alone = make_case(tmp_path / f"a{k}", op, A, 0.8, nx, steps, pq=pq)
        prog = "itlbm_incl" if pq else "itlbm_ops"
        assert run(BIN / prog, alone).returncode == 0
        names = ["inclinada.dat"] if pq else ["laplace.dat", "iso.dat", "galilean.dat"]
        # the final fields: perfil.dat of a strip (Imm_INCL.cpp:101, :162), the rho_R / rho_B / vel_
        # files of a drop at its last step (Imm_OPS.cpp:357-364)
        names += ["perfil.dat"] if pq else [f"rho_R{steps - 1}.vtk", f"rho_B{steps - 1}.vtk", f"vel_{steps - 1}.vtk"]
        for n in names:
            assert (dirs[k] / n).read_bytes() == (alone / n).read_bytes(), (k, n)
        ra = (dirs[k] / "resumo.dat").read_text().splitlines()
        rb = (alone / "resumo.dat").read_text().splitlines()
        assert ra[0] == rb[0] and ra[1].split()[:-1] == rb[1].split()[:-1]  # all but the MLUPS column
    # the analisar_lote.py table rows, appended as each case retired
    import csv
    with open(spool / "resumo_gota.csv", newline="") as f:
        gota = {r["pasta"]: r for r in csv.DictReader(f)}
    with open(spool / "resumo_incl.csv", newline="") as f:
        incl = {r["pasta"]: r for r in csv.DictReader(f)}
    n_strips = sum(1 for c in cases if c[4])
    assert len(gota) == len(cases) - n_strips and len(incl) == n_strips
    for k, c in enumerate(cases):
        row = (incl if c[4] else gota)[f"s{k}"]
        assert row["rotulo"] == f"s{k}" and row["estado"] == "estavel"
    import json
    stats = json.loads((spool / "serve_stats.json").read_text())
    assert stats["completed"] == len(cases) and stats["invalid"] == 1 and stats["p99_s"] > 0


def test_fold_word_served_and_alone(tmp_path):
    """ITLBM_PRECISION=fold picks the nine-class FP32 storage through the server and through itlbm_ops
    alike (the same bytes), and its Laplace jump, tension and area radius stay within the FP32 bars of
    the FP64 run of the same folder."""
    from test_dropin import _rows
    spool = tmp_path / "spool"
    spool.mkdir()
    server = subprocess.Popen([str(BIN / "itlbm_serve"), str(spool), "--idle-exit", "2", "--chunk", "250"],
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        served = make_case(tmp_path / "served", "P3 0.5", 0.225, 0.8, 48, 1001)
        r = submit(served, spool, prec="fold")
        assert r.returncode == 0, r.stderr
    finally:
        server.wait(timeout=120)
    alone = make_case(tmp_path / "alone", "P3 0.5", 0.225, 0.8, 48, 1001)
    r = run(BIN / "itlbm_ops", alone, {"ITLBM_PRECISION": "fold"})
    assert r.returncode == 0 and "nove classes" in r.stdout
    assert (served / "laplace.dat").read_text() == (alone / "laplace.dat").read_text()
    ref = make_case(tmp_path / "fp64", "P3 0.5", 0.225, 0.8, 48, 1001)
    assert run(BIN / "itlbm_ops", ref).returncode == 0
    rows_f, rows_d = _rows(alone / "laplace.dat"), _rows(ref / "laplace.dat")
    assert len(rows_f) == len(rows_d) == 3
    for a, b in zip(rows_f[1:], rows_d[1:]):  # steps 500 and 1000
        assert abs(float(a[6]) - float(b[6])) <= 5e-3 * abs(float(b[6]))  # delta_p
        assert abs(float(a[7]) - float(b[7])) <= 5e-3 * abs(float(b[7]))  # sigma
        assert abs(float(a[1]) - float(b[1])) <= 2e-4 * float(b[1])  # raio_area
