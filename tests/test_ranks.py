"""Multi-rank host plumbing of bench.py on CPU: two gloo ranks.

`python bench.py --gpus N` runs one independent system per rank (weak scaling,
no data-path collective); the ranks meet only at barriers around the timed
region and in a max over ranks of the timed durations.  These tests run that
plumbing as two processes over gloo, the way torchrun starts them.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, os, sys, time
    sys.path.insert(0, {root!r})
    import bench
    R = bench.Ranks(int(os.environ["LOCAL_RANK"]))
    R.barrier()
    t = 0.25 * (R.rank + 1)             # this rank's timed duration
    worst = R.max(t)
    # every rank takes the same collective steps in the same order
    R.barrier()
    again = R.max(-float(R.rank))
    R.close()
    print(json.dumps({{"rank": R.rank, "ws": R.ws, "max": worst, "max2": again}}))
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(n):
    port = _free_port()
    code = CHILD.format(root=ROOT)
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e[-2000:]
        out.append(json.loads(o.strip().splitlines()[-1]))
    return sorted(out, key=lambda d: d["rank"])


def test_two_gloo_ranks_barrier_and_max():
    res = _run_ranks(2)
    assert [d["rank"] for d in res] == [0, 1]
    assert all(d["ws"] == 2 for d in res)
    # the timed duration every rank reports is the slowest rank's
    assert all(d["max"] == pytest.approx(0.5) for d in res)
    assert all(d["max2"] == pytest.approx(0.0) for d in res)


def test_single_rank_is_a_no_op(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    R = bench.Ranks(0)
    assert (R.ws, R.rank) == (1, 0)
    R.barrier()
    assert R.max(3.5) == 3.5
    R.close()


def _bench_reference(rank, ws):
    env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws),
               CUDA_VISIBLE_DEVICES="")
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--workload", "argon4k", "--steps", "2", "--warmup", "1", "--gpus", str(ws)],
                          env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)


def test_reference_arm_rank0_reports_other_ranks_exit_quietly():
    """The reference arm under torchrun: rank 0 alone times the reference's CPU
    implementation and prints the line; every other rank exits 0 without work."""
    r1 = _bench_reference(1, 2)
    assert r1.returncode == 0, r1.stderr[-2000:]
    assert r1.stdout.strip() == ""
    r0 = _bench_reference(0, 2)
    assert r0.returncode == 0, r0.stderr[-2000:]
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "atom-steps/s"
    assert line["n_gpus"] == 2 and line["value"] > 0
    assert line["config"]["workload"] == "argon4k"
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "atom-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
