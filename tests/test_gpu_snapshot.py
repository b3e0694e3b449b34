"""Case snapshots (no counterpart in the reference, which restarts an interrupted batch from step 0,
rodar_lote.py:5-7): a case saved after some steps and restored, alone or in a batch, must go on to
give the same bits as the uninterrupted run; the server, with --snapshots, resumes a case folder from
its snapshot and writes the same files as a run that was never interrupted."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from test_dropin import BIN, make_case, run

pytestmark = pytest.mark.gpu


def desc(itlbm, nx, tipo, prec, geometry=0, p=1, q=0, v0=0.0):
    op = itlbm.make_op(tipo, 0.5, 1.569988)
    return itlbm.desc(nx, nx, op, tau=0.8, A_fact=0.225 if tipo < 11 else 0.1, precision=prec,
                      geometry=geometry, p=p, q=q, v0=v0, k_profile=2.0 * math.log(9.0) / 3.45)


@pytest.mark.parametrize("nx,tipo,prec,geometry,v0", [(64, 3, 0, 0, 0.05), (70, 12, 1, 0, 0.0),
                                                       (48, 11, 0, 1, 0.0), (53, 13, 1, 0, 0.02),
                                                       (50, 13, 2, 0, 0.01), (44, 11, 2, 1, 0.0)])
def test_case_resumes_bit_for_bit(gpu, tmp_path, nx, tipo, prec, geometry, v0):
    d = desc(gpu, nx, tipo, prec, geometry, p=2, q=1, v0=v0)
    with gpu.Case(d) as full:
        full.step(349)
        full.step(1, keep_aux=True)
        ref = full.read_pops(0)
        ref_diag = full.diag_strip(349).as_dict() if geometry else full.diag_drop(349).as_dict()
    snap = tmp_path / "estado.bin"
    with gpu.Case(d) as part:
        part.step(211)
        part.save(snap)
    info_d, info_s = gpu.CaseDesc(), C.c_longlong()
    gpu.check(gpu.lib().itlbm_snapshot_info(str(snap).encode(), C.byref(info_d), C.byref(info_s)), "info")
    assert info_s.value == 211 and info_d.nx == nx and info_d.precision == prec
    c = gpu.Case.load(snap)
    try:
        assert c.steps_done == 211
        c.step(138)
        c.step(1, keep_aux=True)
        got = c.read_pops(0)
        assert np.array_equal(ref[0], got[0]) and np.array_equal(ref[1], got[1])
        got_diag = c.diag_strip(349).as_dict() if geometry else c.diag_drop(349).as_dict()
        for k, v in ref_diag.items():
            assert v == got_diag[k] or (v != v and got_diag[k] != got_diag[k]), k
    finally:
        c.close()


def test_bad_snapshots_are_refused(gpu, tmp_path):
    h = C.c_void_p()
    assert gpu.lib().itlbm_case_load(str(tmp_path / "none.bin").encode(), C.byref(h)) == -9  # ITLBM_E_IO
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not a snapshot at all" * 20)
    assert gpu.lib().itlbm_case_load(str(bad).encode(), C.byref(h)) == -8  # ITLBM_E_PARSE
    with gpu.Case(desc(gpu, 40, 3, 0)) as c:
        c.step(5)
        c.save(tmp_path / "ok.bin")
    data = (tmp_path / "ok.bin").read_bytes()
    (tmp_path / "short.bin").write_bytes(data[: len(data) // 2])
    assert gpu.lib().itlbm_case_load(str(tmp_path / "short.bin").encode(), C.byref(h)) == -8


def diag_rows(itlbm, b):
    rows = {}
    for _ in range(100):
        b.advance()
        for e in b.poll():
            if e.kind == itlbm.EV_DIAG:
                rows[(e.tag, e.step)] = e.drop.as_dict() if e.geometry == 0 else e.strip.as_dict()
        if b.stats().active == 0 and b.stats().pending == 0:
            break
    return rows


def test_batch_resumes_bit_for_bit(gpu, tmp_path):
    specs = [desc(gpu, 64, 3, 0), desc(gpu, 80, 12, 1), desc(gpu, 48, 13, 0, geometry=1, p=1, q=1)]
    with gpu.Batch(chunk=200, diag_every=500) as b:
        for k, d in enumerate(specs):
            b.submit(d, 1201, k)
        ref = diag_rows(gpu, b)
    # the same cases, interrupted after their diagnostic at step 500 and resumed in a new batch
    with gpu.Batch(chunk=200, diag_every=500) as b:
        for k, d in enumerate(specs):
            b.submit(d, 1201, k)
        seen = set()
        for _ in range(20):
            b.advance()
            for e in b.poll():
                if e.kind == gpu.EV_DIAG and e.step == 500:
                    b.save(e.tag, tmp_path / f"c{e.tag}.bin")
                    seen.add(e.tag)
            if len(seen) == len(specs):
                break
    with gpu.Batch(chunk=200, diag_every=500) as b:
        for k in range(len(specs)):
            b.submit_saved(tmp_path / f"c{k}.bin", 1201, k)
        got = diag_rows(gpu, b)
    for k in range(len(specs)):
        for step in (1000, 1200):
            a, g = ref[(k, step)], got[(k, step)]
            for key, v in a.items():
                assert v == g[key] or (v != v and g[key] != g[key]), (k, step, key)
        assert (k, 500) not in got  # resumed after its step-500 diagnostic


def test_server_resumes_a_folder(tmp_path):
    """A case served with --snapshots for 1001 steps, then asked for 2001: the server resumes from its
    last snapshot (step 500) and the folder ends with the files of a direct 2001-step run."""
    spool = tmp_path / "spool"
    spool.mkdir()
    a = make_case(tmp_path / "a", "P3 0.5", 0.225, 0.8, 48, 1001)
    env_serve = [str(BIN / "itlbm_serve"), str(spool), "--idle-exit", "2", "--chunk", "250", "--snapshots",
                 "--fp64"]

    def serve_once():
        server = subprocess.Popen(env_serve, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        try:
            env = dict(os.environ, ITLBM_SPOOL=str(spool), ITLBM_PRECISION="fp64", ITLBM_SUBMIT_TIMEOUT="250")
            r = subprocess.run([str(BIN / "itlbm_submit")], cwd=a, capture_output=True, text=True, timeout=300,
                               env=env)
            assert r.returncode == 0, r.stderr
        finally:
            _, err = server.communicate(timeout=120)
        return err

    err = serve_once()
    assert (a / "estado_itlbm.bin").exists() and (a / "estado_itlbm.run").exists(), (err, sorted(os.listdir(a)))
    make_case(a, "P3 0.5", 0.225, 0.8, 48, 2001)  # the same case, asked for more steps
    serve_once()
    direct = make_case(tmp_path / "d", "P3 0.5", 0.225, 0.8, 48, 2001)
    assert run(BIN / "itlbm_ops", direct).returncode == 0
    for n in ("laplace.dat", "iso.dat", "galilean.dat"):
        assert (a / n).read_text() == (direct / n).read_text(), n
    ra, rd = (a / "resumo.dat").read_text().splitlines(), (direct / "resumo.dat").read_text().splitlines()
    assert ra[0] == rd[0] and ra[1].split()[:-1] == rd[1].split()[:-1]
