"""bench.py host paths on the CPU: the reduction over ranks with two gloo ranks, and the
reference arm's JSON line (the oracle port on a small workload)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, p = bench.reduce_over_ranks(1.5 + rank, 10 * (rank + 1), "cpu")
        out.put((rank, t, p))
    finally:
        dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [r[0] for r in res] == [0, 1]
    for _, t, p in res:
        assert t == 2.5 and p == 30.0  # max of (1.5, 2.5); sum of (10, 20)


def test_reference_arm_prints_its_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--workload", "single_aperture_2grid"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "particle-pushes/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_traffic_summaries_parse_per_workload():
    """Each headline workload has its own ncu traffic summary with a kernel-source hash and the
    DRAM bytes per particle of both step kernels; bench.traffic_table reads it (or reports it
    stale when the kernel sources changed since the capture)."""
    sys.path.insert(0, ROOT)
    import bench
    for name in ("long_erosion_3grid", "large_aperture_3grid"):
        with open(bench.TRAFFIC_PROFILES[name]) as f:
            text = f.read()
        assert "kernel_source_sha:" in text
        assert text.count("dram_bytes_per_particle:") == 2
        table, note = bench.traffic_table(name)
        if note.startswith("stale"):
            assert table == {}
        else:
            assert set(table) == {"k_ion_step", "k_ele_step"} and all(v >= 41.0 for v in table.values())
    assert bench.traffic_table("no_such_workload") == ({}, "no ncu traffic summary for no_such_workload")
