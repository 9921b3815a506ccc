"""The N > 1 path of bench.py on the CPU with gloo, world size 2 (the update is
replicas only: no data-path collective).

  * Dist: the max over ranks and the barrier that bracket every timed region;
  * the reference arm under torchrun: rank 0 alone runs the CPU restatement and
    prints one JSON line with n_gpus 2; rank 1 exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import bench
d = bench.Dist(2)
got = d.max(float(d.rank) + 1.5)
d.barrier()
print(json.dumps({{"rank": d.rank, "world": d.world, "max": got}}), flush=True)
d.close()
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_dist_max_and_barrier_over_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=str(ROOT))], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert all(o["world"] == 2 and o["max"] == 2.5 for o in outs)


def test_reference_arm_on_two_ranks_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["config"]["parallelism"] == "replicas"
