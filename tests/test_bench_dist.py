"""bench.py's multi-process plumbing (one process per GPU under torchrun):
barrier, max and sum over ranks, exercised with two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

CHILD = r"""
import sys
sys.path.insert(0, {root!r})
import bench
d = bench.Dist(2)
assert d.world == 2
d.barrier()
r = d.rank
mx = d.max(10.0 + r)          # per-rank device time: the job time is the slowest
sm = d.sum(1000 * (r + 1))    # per-rank lattice updates: the job total
d.barrier()
d.close()
print("rank", r, mx, sm)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_max_and_sum_over_gloo():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(out)
    for rank, out in enumerate(outs):
        assert ("rank %d 11.0 3000.0" % rank) in out, out


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
