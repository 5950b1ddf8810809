"""bench.py's multi-process plumbing on CPU: two gloo ranks (127.0.0.1).

With N > 1 every rank runs a replica; the ranks meet only in a barrier and
in the max / sum of their timings.  The reference arm runs on rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CHILD = textwrap.dedent("""
    import json, os, sys, argparse
    sys.path.insert(0, os.environ["HGM_TEST_ROOT"])
    import bench
    d = bench.Dist()
    r = d.rank
    d.barrier()
    mx = d.max(float(r + 1) * 10.0)
    sm = d.sum(float(r + 1))
    args = argparse.Namespace(workload="nonexistent", steps=1, warmup=0, requests=0, qubits=0,
                              metric_name="x")
    ref = bench.reference_arm(args, d)
    print("RESULT " + json.dumps({"rank": r, "world": d.world, "max": mx, "sum": sm, "ref": ref}), flush=True)
    d.close()
""")


def test_two_gloo_ranks_reduce_and_reference_on_rank0():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), HGM_TEST_ROOT=str(ROOT))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        so, se = p.communicate(timeout=180)
        assert p.returncode == 0, se
        line = [l for l in so.splitlines() if l.startswith("RESULT ")][0]
        out.append(json.loads(line[len("RESULT "):]))
    out.sort(key=lambda d: d["rank"])
    assert [d["world"] for d in out] == [2, 2]
    assert all(d["max"] == 20.0 for d in out)          # max over ranks
    assert all(d["sum"] == 3.0 for d in out)           # units of all ranks
    assert out[0]["ref"]["impl"] == "reference"        # rank 0 answers for the reference arm
    assert "unavailable" in out[0]["ref"]
    assert out[1]["ref"] is None                       # the other ranks do no work
