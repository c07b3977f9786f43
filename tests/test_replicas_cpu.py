"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the path is
replicas only (every rank runs the whole per-GPU workload on its own data), so
the only cross-rank steps are the barrier around the timed region and the
max-over-ranks time that the whole-job rate divides by."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_max_time():
    port = _free_port()
    script = textwrap.dedent("""
        import os, sys, json
        sys.path.insert(0, %r)
        import torch.distributed as dist
        import bench
        rank = int(os.environ["RANK"])
        dist.init_process_group("gloo", rank=rank, world_size=2)
        bench.barrier(2)
        t = bench.max_over_ranks(2, 1.5 + rank)        # rank 1 is the slow one
        units = 512 * 2                                   # replicas: each rank did 512 rotations
        print(json.dumps({"rank": rank, "max": t, "rate": units / t}))
        bench.barrier(2)
        dist.destroy_process_group()
    """ % ROOT)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", script], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    import json
    res = [json.loads(o.strip().splitlines()[-1]) for o, _ in outs]
    assert all(r["max"] == 2.5 for r in res)
    assert all(abs(r["rate"] - 1024 / 2.5) < 1e-9 for r in res)
