"""The N > 1 path of bench.py on CPU: two gloo ranks, as torchrun would start them.

Cases are independent, so N GPUs run N replicas with no data-path collective; the only collectives
are the barrier and the reductions of the result: every rank's node updates over the slowest rank's
device time.  The reference arm runs on rank 0 only; the other ranks exit 0 without work."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(REPO))
    import bench
    import torch.distributed as dist
    w, r, local = bench.setup_dist("gloo")
    # rank r processed (r + 1) million node updates in 10 (r + 1) ms
    mlups, ms_max = bench.replica_mlups((r + 1) * 1e6, 10.0 * (r + 1), w)
    bench.barrier(w)
    Path(out_dir, f"r{r}.json").write_text(json.dumps({"world": w, "local": local, "mlups": mlups,
                                                       "ms_max": ms_max}))
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r, x in enumerate(res):
        assert x["world"] == 2 and x["local"] == r
        assert x["ms_max"] == 20.0                      # max over ranks
        assert x["mlups"] == pytest.approx(3e6 / 20e-3 / 1e6)  # sum of updates / slowest time


def _ref_rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(REPO))
    import contextlib
    import io

    import bench
    buf = io.StringIO()
    args = type("A", (), dict(gpus=world, steps=1, warmup=3, workload="batch600"))()
    with contextlib.redirect_stdout(buf):
        rc = bench.run_reference(args)
    Path(out_dir, f"r{rank}.txt").write_text(f"{rc}\n{buf.getvalue()}")


def test_reference_arm_rank0_only(tmp_path):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle
    if not oracle.REF_DIR.joinpath("libref_ops_fast.so").exists():
        pytest.skip("oracle/_ref not built")
    world = 2
    mp.start_processes(_ref_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    rc0, out0 = (tmp_path / "r0.txt").read_text().split("\n", 1)
    rc1, out1 = (tmp_path / "r1.txt").read_text().split("\n", 1)
    assert rc0 == "0" and rc1 == "0"
    assert out1.strip() == ""
    line = json.loads(out0.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
