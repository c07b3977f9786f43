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


def test_bench_gpus_flag_launches_ranks():
    """`bench.py --gpus 2` launches two ranks itself (torch.distributed.run on
    127.0.0.1) and the printed line carries n_gpus = 2. The reference arm runs
    on the host cores, so this runs on CPU: rank 0 measures and prints, rank 1
    exits without work."""
    import json
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "multiply", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-3000:]
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["impl"] == "reference"


def test_bench_rejects_mismatched_world_size():
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "multiply", "--steps", "1"], env=env, capture_output=True, text=True,
                       timeout=300, cwd=ROOT)
    assert r.returncode != 0 and "WORLD_SIZE=3" in (r.stderr + r.stdout)
