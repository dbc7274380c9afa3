"""The N > 1 path of bench.py on two gloo ranks on the CPU: the timing
collectives (max over ranks, barrier) and the reference arm's rule that rank 0
alone prints one JSON line while the other ranks exit without output."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import os, sys, io, json, contextlib
sys.path.insert(0, {root!r})
import bench
class A: impl = "reference"
world, rank, local, pg = bench.dist_setup(A())
out = {{"world": world, "rank": rank}}
out["max"] = bench.max_over_ranks(pg, 1.5 + rank, local)
bench.barrier(pg, local)
pg.barrier()
pg.destroy_process_group()
# the reference arm under torchrun: only rank 0 prints
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    sys.argv = ["bench.py", "--impl", "reference", "--workload", "adi", "--steps", "3", "--warmup", "3",
                "--gpus", str(world)]
    bench.main()
out["printed"] = buf.getvalue()
print("RESULT " + json.dumps(out))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(240)
def test_two_gloo_ranks():
    port = free_port()
    code = RANK_SCRIPT.format(root=ROOT)
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=200)
        assert p.returncode == 0, e[-2000:]
        line = [l for l in o.splitlines() if l.startswith("RESULT ")][-1]
        outs.append(json.loads(line[len("RESULT "):]))
    for o in outs:
        assert o["world"] == 2 and o["max"] == 2.5
    rank0 = next(o for o in outs if o["rank"] == 0)
    rank1 = next(o for o in outs if o["rank"] == 1)
    printed = [json.loads(l) for l in rank0["printed"].splitlines() if l.strip()]
    assert len(printed) == 1 and printed[0]["impl"] == "reference"
    assert rank1["printed"].strip() == ""
