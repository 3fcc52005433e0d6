"""Host-side multi-rank logic of bench.py on CPU: two gloo ranks (spawned
processes) check the max-over-ranks timing reduction and the barrier; the
reference arm runs on rank 0 alone and prints one JSON line there."""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as td

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        v = bench.max_over_ranks(1.5 + rank, None)
        bench.barrier(None)
        v2 = bench.max_over_ranks(10.0 - rank, "cpu")
        q.put((rank, v, v2))
    finally:
        td.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.5, 10.0), (1, 2.5, 10.0)]


def test_helpers_single_process():
    import bench

    assert bench.max_over_ranks(3.25) == 3.25
    bench.barrier(None)  # no process group: no-op
    a = bench.parse(["--steps", "2", "--warmup", "3", "--no-extras", "--mesh", "8x4x4"])
    assert a.steps == 2 and a.warmup == 3 and a.no_extras and bench.mesh_dims(a.mesh) == (8, 4, 4)
    assert bench.parse([]).impl == "ours"


def test_reference_arm_rank0_only(monkeypatch, capsys):
    import bench

    args = bench.parse(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                        "--mesh", "6x3x3", "--cpu-iters", "2"])
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    bench.run_reference(args)
    assert capsys.readouterr().out == ""  # rank 1 exits without work
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("LOCAL_RANK", "0")
    bench.run_reference(args)
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["higher_is_better"] is False
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["value"] == line["value"]


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
