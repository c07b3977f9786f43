"""Throughput benchmark of the B200 RNS-CKKS hot path.

python bench.py [--gpus N] [--steps K] [--warmup W] [--workload rotation|ntt|multiply|ccmm|fft2|park] [--park-n n] [--impl reference]

Workload "rotation" (default): hoisted key-switched Galois rotations at
N=2^16 over 24 Q limbs of 50-bit primes and 3 auxiliary 60-bit primes (the
reference's prime search), the reference's bounded hybrid-QP gadget with base
2^32 (38 digits, tests/r30_9a_13_hybrid_65536.rs default), 16 ciphertexts each
rotated by the same 32 Galois steps (powers of two 1..2^14 and odd steps
3..35) sharing one decomposition per ciphertext. One step = all 512
rotations; outputs are word-for-word the reference algorithm's. Metric:
rotations per second. The line also carries, measured in the same run:
  parity      the CPU baseline runs the oracle on the timed batch's own
              ciphertexts and (downloaded) keys and its outputs are compared
              word for word with the GPU's, plus one fresh encryption decoded
              on both sides (decoded_error);
  ccmm        the metric's second half: one 64 x 64 structured CCMM at N=2^15
              (the "ccmm" workload below; 3 timed after 3 warm-up products)
              with its own roofline, e2e, parity and CPU baseline
              (--no-ccmm leaves it out);
  park        Park Mod-PP-MM at n = 4096 (the "park" workload below; 5 timed
              after 3 warm-up products) with its own roofline, e2e, parity,
              CUDA-core form and CPU baseline (--no-park leaves it out);
  plain_gpu   the plain GPU forms of the same rotations.

Workload "ntt": batched forward + inverse negacyclic NTT at N=2^16 over 32
limbs of 50-bit primes q = 1 mod 2N (the reference's prime search), 64
polynomials per launch, residues uniform in [0, q). One step = one forward and
one inverse transform of the whole batch. Metric: limb-polynomial transforms
per second (forward and inverse each count once).

Workload "ccmm": structured encrypted matrix product of two 64 x 64 matrices
of ciphertexts (one per entry) at N=2^15 over 14 x 50-bit limbs with the
bounded relinearization key (base 2^20): sum of 64 tensors per output entry,
relinearize, rescale. One step = one 64 x 64 CCMM. Metric: CCMM per second.

Workload "fft2": encrypted 2-D FFT of eight 256 x 256 real images, two
ciphertexts per image at N=2^16 (24 x 50-bit Q, 3 x 60-bit P), with the
radix-4 diagonal-rotation schedule: 4 row and 4 column stages, each
sum(diagonal * rotation) + rescale. One step = 8 images. Metric: images/s.

Workload "park": the Park Mod-PP-MM (ccmm/park.rs:1634-1647) of two 4096 x 4096
u64 residue matrices mod 0x7ffff6001 (the largest size and the modulus of the
reference's characterization binary). One step = one product. Metric: products/s.

Workload "multiply": the plain CKKS chain at N=2^12 (q = 60 + 40 + 40 bits,
P = 60 bits, the reference's prime search): HMult -> bounded relinearization
(base 2^20) -> rescale -> key-switched rotation by one slot, for 64
ciphertext pairs. One step = 64 chains. Metric: chains per second.

One JSON line on rank 0. `--gpus N` runs N independent replicas, one process
per GPU (launched through torch.distributed.run when no torchrun environment is
set; the path shards into independent polynomials/ciphertexts, with no
collective on the data path): value = units of all ranks / max-over-ranks
time. CPU baselines and parity checks run at N=1.
`--impl reference` times the CPU restatement of the reference algorithm
(oracle/, the reference itself is Rust and cannot be built here) on the host
cores with every thread, on the same workload and metric.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ccmm-rs_b200"))

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def bf16_peak():
    """Dense bf16 TF/s of this pool's B200s (burst figure) and where it came from."""
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return FALLBACK_BF16_TFLOPS, "fallback"


# ------------------------------------------------------------ clocks sampler
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # let nvidia-smi start up (and take its first sample) before the timed
            # region, so its start-up does not overlap the timed launches
            t = time.time()
            while not self.lines and time.time() - t < 5.0 and self.proc.poll() is None:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def count_launches(fn):
    """Kernel launches of one call of fn (counted by the CUDA profiler hooks
    torch ships, outside every timed region); None when tracing is unavailable."""
    try:
        import torch
        from torch.profiler import ProfilerActivity, profile
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        n = 0
        for e in prof.events():
            name = getattr(e, "name", "") or ""
            if str(getattr(e, "device_type", "")).endswith("CUDA") and not name.startswith(("Memcpy", "Memset")):
                n += 1
        return n if n > 0 else None
    except Exception:
        return None


# --------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------- NTT
NTT_LOG_N, NTT_LIMBS, NTT_POLYS, NTT_BITS = 16, 32, 64, 50


def ntt_primes():
    # the reference's prime search: descending from 2^50-1 in steps of 2N
    # (security/p6a/generate_candidates.py:53-73)
    sys.path.insert(0, os.path.join(ROOT, "ccmm-rs_b200"))
    import ckks_b200.params as params
    return params.primes_below_bits(NTT_BITS, 1 << NTT_LOG_N, NTT_LIMBS)


def ntt_config():
    return {"workload": "batched NTT+iNTT, N=2^16, 32 x 50-bit limbs, 64 polys/launch",
            "log_n": NTT_LOG_N, "limbs": NTT_LIMBS, "polys_per_launch": NTT_POLYS,
            "l2": "inputs (1.07 GB) larger than L2", "parallelism": "replicas"}


def bench_ntt_gpu(args, world, rank, local):
    import torch
    import ckks_b200 as cb
    dev = torch.device("cuda", local)
    n = 1 << NTT_LOG_N
    primes = ntt_primes()
    ctx = cb.Context(NTT_LOG_N, primes)
    # NTT tile choices timed on this workload's batch (outside the timed region)
    tuning = ctx.autotune(limbs=NTT_LIMBS, polys=NTT_POLYS)
    rng = np.random.default_rng(1234 + rank)
    host = np.stack([rng.integers(0, q, (NTT_POLYS, n), dtype=np.uint64) for q in primes], axis=1)
    data = cb.as_u64_tensor(host, dev)
    tmp = torch.empty_like(data)
    st = torch.cuda.current_stream()

    def step():
        ctx.ntt_forward(data, out=tmp)
        ctx.ntt_inverse(tmp, out=data)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # per-kernel timing of one forward transform (both passes) for the roofline
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    fwd_ms = []
    for _ in range(3):
        ev[0].record(st)
        ctx.ntt_forward(data, out=tmp)
        ev[1].record(st)
        torch.cuda.synchronize()
        fwd_ms.append(ev[0].elapsed_time(ev[1]))
        ctx.ntt_inverse(tmp, out=data)
    torch.cuda.synchronize()

    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        step()
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    units = 2 * NTT_POLYS * NTT_LIMBS * args.steps * world
    value = units / (ms_max / 1000.0)

    # roofline: forward NTT = 16 N bytes per limb-poly (read + write)
    alg_bytes = 16 * n * NTT_POLYS * NTT_LIMBS
    fwd = float(np.median(fwd_ms))
    peak, kind = peaks()
    achieved = alg_bytes / (fwd / 1000.0) / 1e9

    # end to end through the C ABI host-buffer call (pinned host memory)
    pinned_in = torch.from_numpy(host.view(np.int64)).pin_memory()
    pinned_out = torch.empty_like(pinned_in).pin_memory()
    hin = pinned_in.numpy().view(np.uint64)
    hout = pinned_out.numpy().view(np.uint64)
    import ctypes
    lib = cb.lib()
    e2e_steps = max(1, min(args.steps, 5))
    ctx.ntt_forward_host(hin)  # warm
    barrier(world)
    t = time.perf_counter()
    for _ in range(e2e_steps):
        rc = lib.ckks_ntt_forward_host(ctx.handle, hin.ctypes.data_as(cb.u64p), hout.ctypes.data_as(cb.u64p),
                                       NTT_POLYS, 0, NTT_LIMBS)
        cb.check(rc)
    e2e_s = max_over_ranks(world, (time.perf_counter() - t))
    e2e_value = NTT_POLYS * NTT_LIMBS * e2e_steps * world / e2e_s

    line = {
        "metric": "limb-polynomial NTT transforms/s (N=2^16, 50-bit limbs)", "value": value,
        "unit": "limb-NTT/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded uniform residues)",
        "config": dict(ntt_config(), autotune=tuning.strip().splitlines()),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": kind,
                     "kernel": "forward NTT (pass1+pass2), %d limb-polys/launch" % (NTT_POLYS * NTT_LIMBS),
                     "kernel_ms": fwd},
        "e2e": {"value": e2e_value, "unit": "limb-NTT/s", "h2d_bytes_per_step": int(host.nbytes),
                "d2h_bytes_per_step": int(host.nbytes), "path": "ckks_ntt_forward_host"},
        "gpu_launches": 4 * args.steps, "clocks": clk,
    }
    return line


def ntt_cpu_sample(threads, seconds_target=10.0):
    """Times the oracle NTT (restated reference radix-2 Shoup NTT) on host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle, P, arr
    import concurrent.futures as cf
    o = Oracle()
    n = 1 << NTT_LOG_N
    primes = ntt_primes()
    rng = np.random.default_rng(99)
    per_thread = np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in primes])  # 32 limbs
    moduli = arr(primes)
    bufs = [per_thread.copy() for _ in range(threads)]

    def work(b):
        o.L.oracle_ntt_forward(P(moduli), NTT_LIMBS, n, P(b), 1)
        o.L.oracle_ntt_inverse(P(moduli), NTT_LIMBS, n, P(b), 1)

    work(bufs[0])
    t = time.perf_counter()
    rounds = 0
    with cf.ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t < seconds_target:
            list(ex.map(work, bufs))
            rounds += 1
    dt = time.perf_counter() - t
    units = rounds * threads * 2 * NTT_LIMBS
    return units / dt, "%d rounds x %d threads x 32 limbs x (fwd+inv) at N=2^16" % (rounds, threads)


def reference_arm(args, world, rank):
    if rank != 0:
        return None
    if args.workload == "fft2":
        threads = os.cpu_count() or 1
        vals, sample = [], None
        for i in range(1 + args.steps):
            v, sample = fft2_cpu_sample(threads)
            if i >= 1:
                vals.append(v)
        value = float(np.median(vals))
        return {
            "metric": "encrypted 256x256 FFT2 images/s (N=2^16, 24 limbs, radix-4 schedule, bit-exact)",
            "value": value, "unit": "images/s", "n_gpus": world, "steps": args.steps, "warmup": 1,
            "ms_per_step": 1000.0 * FFT2_IMAGES / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts)",
            "config": fft2_config(), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "images/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    if args.workload == "ccmm":
        threads = os.cpu_count() or 1
        vals, sample = [], None
        for i in range(1 + args.steps):
            v, sample = ccmm_cpu_sample(threads)
            if i >= 1:
                vals.append(v)
        value = float(np.median(vals))
        return {
            "metric": "64x64 structured CCMM/s (N=2^15, 14 limbs, both operands encrypted, bit-exact)",
            "value": value, "unit": "CCMM/s", "n_gpus": world, "steps": args.steps, "warmup": 1,
            "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64", "data": "synthetic (seeded uniform ciphertext residues)", "config": ccmm_config(),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "CCMM/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "CCMM/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    if args.workload == "multiply":
        threads = os.cpu_count() or 1
        vals, sample = [], None
        for i in range(args.warmup + args.steps):
            v, sample = mul_cpu_sample(threads, pairs=4 * threads)
            if i >= args.warmup:
                vals.append(v)
        value = float(np.median(vals))
        return {
            "metric": "HMult+relinearize+rescale+rotate chains/s (N=2^12, 3 limbs, bit-exact)", "value": value,
            "unit": "chains/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * MUL_PAIRS / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts)",
            "config": mul_config(), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "chains/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "chains/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    if args.workload == "rotation":
        return reference_rotation(args, world)
    if args.workload == "park":
        threads = os.cpu_count() or 1
        vals, sample = [], None
        for i in range(args.warmup + args.steps):
            v, sample = park_cpu_sample(threads, args.park_n)
            if i >= args.warmup:
                vals.append(v)
        value = float(np.median(vals))
        return {
            "metric": park_metric(args.park_n), "value": value, "unit": "products/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform residues)",
            "config": park_config(args.park_n), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "products/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    threads = os.cpu_count() or 1
    per_step = []
    sample = None
    for i in range(args.warmup + args.steps):
        v, sample = ntt_cpu_sample(threads, seconds_target=max(2.0, 20.0 / max(1, args.steps + args.warmup)))
        if i >= args.warmup:
            per_step.append(v)
    value = float(np.median(per_step))
    return {
        "metric": "limb-polynomial NTT transforms/s (N=2^16, 50-bit limbs)", "value": value,
        "unit": "limb-NTT/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * 2 * NTT_POLYS * NTT_LIMBS / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform residues)",
        "config": ntt_config(), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "limb-NTT/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "limb-NTT/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def reference_rotation(args, world):
    """Reference arm of the rotation workload: the oracle's restatement of the
    reference's hoisted rotation on every host core. Keys are made once; each
    timed step is a real sample of one ciphertext per thread x 2 Galois keys
    (the decomposition is shared by the keys of a ciphertext, as in the
    reference's automorphism_hoisted; per key the reference re-transforms every
    digit, so the rate hardly depends on the key count: the line records the
    measured per-key and per-decomposition cost). A 1-thread figure follows."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle, arr
    import concurrent.futures as cf
    o = Oracle()
    threads = os.cpu_count() or 1
    n = 1 << ROT_LOG_N
    q = arr(o.primes_below_bits(ROT_QBITS, n, ROT_L))
    p = arr(o.primes_below_bits(ROT_PBITS, n, ROT_K))
    rng = np.random.default_rng(77)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    exps = [int(o.L.oracle_rotation_exponent_left(n, r)) for r in ROT_STEPS[:2]]
    with cf.ThreadPoolExecutor(2) as ex:
        keys = list(ex.map(lambda ik: o.hybrid_key(q, p, secret, ik[1], ROT_BASE_LOG, seed=500 + ik[0]),
                           enumerate(exps)))
    cts = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                    for _ in range(threads)])
    # warm-up: one key per ciphertext (also gives the 1-key cost for the split below)
    v1, _, _ = rot_cpu_sample(threads, 1, keys=keys, exps=exps, cts=cts)
    for _ in range(max(0, args.warmup - 1)):
        rot_cpu_sample(threads, 1, keys=keys, exps=exps, cts=cts)
    vals, samples = [], []
    for _ in range(args.steps):
        v, sample, _ = rot_cpu_sample(threads, 2, keys=keys, exps=exps, cts=cts)
        vals.append(v)
        samples.append(2 * threads / v)
    value = float(np.median(vals))
    # per-thread cost split: t(k keys) = decomposition + k x per-key
    t1, t2 = 1.0 / (v1 / threads), 1.0 / (value / (2 * threads))
    per_key, decomp = t2 - t1, 2 * t1 - t2
    v_1t, sample_1t, _ = rot_cpu_sample(1, 2, keys=keys, exps=exps, cts=cts[:1])
    rots = ROT_NCT * len(ROT_STEPS)
    ccmm = None
    if not args.no_ccmm:
        cv, csample = ccmm_cpu_sample(threads)
        ccmm = {"metric": "64x64 structured CCMM/s (N=2^15, 14 limbs, both operands encrypted, bit-exact)",
                "value": cv, "unit": "CCMM/s", "higher_is_better": True, "config": ccmm_config(),
                "cpu_baseline": {"value": cv, "unit": "CCMM/s", "cores": threads, "kind": "port", "sample": csample}}
    park = None
    if not args.no_park:
        pv, psample = park_cpu_sample(threads, args.park_n)
        park = {"metric": park_metric(args.park_n), "value": pv, "unit": "products/s", "higher_is_better": True,
                "config": park_config(args.park_n),
                "cpu_baseline": {"value": pv, "unit": "products/s", "cores": threads, "kind": "port",
                                 "sample": psample}}
    return {
        "metric": "key-switched rotations/s (N=2^16, 24 limbs, hoisted, bit-exact)", "value": value,
        "unit": "rotations/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * rots / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts)",
        "config": rot_config(), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": threads, "kind": "port", "sample": sample},
        "timed_samples": {"rotations_per_sample": 2 * threads, "seconds": samples,
                          "note": "ms_per_step is the time the measured rate needs for one step of %d rotations "
                                  "(16 ct x 32 keys); each timed sample ran %d rotations" % (rots, 2 * threads)},
        "cost_split_s_per_thread": {"decomposition": decomp, "per_key": per_key,
                                    "rate_at_32_keys": threads * 32 / (decomp + 32 * per_key)},
        "cpu_1thread": {"value": v_1t, "unit": "rotations/s", "cores": 1, "sample": sample_1t},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ccmm": ccmm,
        "park": park,
    }


# -------------------------------------------------------------- rotations
ROT_LOG_N, ROT_L, ROT_K, ROT_QBITS, ROT_PBITS, ROT_BASE_LOG, ROT_NCT = 16, 24, 3, 50, 60, 32, 16
# 32 distinct Galois steps: powers of two 1..2^14 and odd steps 3, 5, .., 35
ROT_STEPS = [1 << i for i in range(15)] + list(range(3, 37, 2))


def rot_config():
    default = (ROT_L == 24 and ROT_NCT == 16 and len(ROT_STEPS) == 32 and ROT_BASE_LOG == 32
               and ROT_LOG_N == 16)
    return {"workload": ("hoisted key-switched rotations, N=2^%d, %dx50-bit Q + 3x60-bit P, bounded hybrid-QP "
                         "gadget base 2^%d, %d ct x %d Galois steps%s"
                         % (ROT_LOG_N, ROT_L, ROT_BASE_LOG, ROT_NCT, len(ROT_STEPS),
                            "" if default else " (reduced profiling size)")),
            "log_n": ROT_LOG_N, "q_limbs": ROT_L, "p_limbs": ROT_K, "base_log": ROT_BASE_LOG,
            "ciphertexts": ROT_NCT, "galois_steps": ROT_STEPS, "scale": "2^50", "secret": "ternary",
            "sigma": 3.2, "l2": "keys and outputs larger than L2", "parallelism": "replicas"}


def bench_rot_gpu(args, world, rank, local):
    import torch
    import ckks_b200 as cb
    import ckks_b200.params as params
    dev = torch.device("cuda", local)
    n = 1 << ROT_LOG_N
    q = params.primes_below_bits(ROT_QBITS, n, ROT_L)
    p = params.primes_below_bits(ROT_PBITS, n, ROT_K)
    ctx = cb.Context(ROT_LOG_N, q, p)
    # NTT tile choices timed on a batch of the rotation's shape (27 limbs), outside the timed region
    tuning = ctx.autotune(limbs=ROT_L + ROT_K, polys=64)
    rng = np.random.default_rng(4321 + rank)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    exps = [ctx.rotation_exponent_left(r) for r in ROT_STEPS]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, ROT_L, ROT_BASE_LOG, k, secret, seed=1000 + i)
            for i, k in enumerate(exps)]
    D, words = keys[0].info()
    # ciphertexts: uniform residues (the distribution of fresh RLWE ciphertexts)
    host = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                     for _ in range(ROT_NCT)])
    cts = cb.as_u64_tensor(host, dev)
    out = torch.empty((ROT_NCT, len(keys), 2, ROT_L, n), dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream()

    def step():
        cb.rotate_hoisted(ctx, keys, cts, out=out)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        step()
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    rots = ROT_NCT * len(keys)
    value = rots * args.steps * world / (ms_max / 1000.0)
    # per-phase device time of one step (outside the timed region)
    _, phases = cb.rotate_hoisted_timed(ctx, keys, cts, out=out)
    torch.cuda.synchronize()
    # roofline of the dominant kernel, the tensor-core key-switch MAC
    # (k_mac_tc): algorithmic bytes per step = every key once per group of 16
    # ciphertexts + the hoisted digit transforms and base transforms of every
    # ciphertext + the accumulators it writes
    key_bytes = words * 8
    LK = ROT_L + ROT_K
    group = 16
    groups = -(-ROT_NCT // group)
    mac_bytes = (groups * len(keys) * key_bytes + ROT_NCT * D * LK * n * 8 + ROT_NCT * ROT_L * n * 8
                 + rots * 2 * LK * n * 8)
    peak, kind = peaks()
    # DRAM traffic per launch: a one-pass ncu capture (dram__bytes_read.sum +
    # dram__bytes_write.sum) of the full-size launch at this shape read 49.954 GB
    # and wrote 14.480 GB against 57.730 GB of algorithmic bytes (the packed key set
    # is 5 % larger than the keys); other shapes scale by the same ratio
    mac_traffic = mac_bytes * (49.954 + 14.480) / 57.730
    mac_ms = phases["key-switch MAC"]
    achieved = mac_bytes / (mac_ms / 1000.0) / 1e9
    ct_bytes = 2 * ROT_L * n * 8
    # end to end through the C ABI host-buffer call (pinned host memory)
    pin_in = torch.from_numpy(host.view(np.int64)).pin_memory()
    pin_out = torch.empty(tuple(out.shape), dtype=torch.int64).pin_memory()
    hin, hout = pin_in.numpy().view(np.uint64), pin_out.numpy().view(np.uint64)
    cb.rotate_hoisted_host(ctx, keys, hin, hout)
    barrier(world)
    e2e_steps = max(1, min(args.steps, 3))
    t = time.perf_counter()
    for _ in range(e2e_steps):
        cb.rotate_hoisted_host(ctx, keys, hin, hout)
    e2e_s = max_over_ranks(world, time.perf_counter() - t)
    # the plain GPU forms of the same rotations, outside the headline timing:
    # one key switch per (ciphertext, key) with no hoisting (ckks_rotate, CUDA-core
    # MAC) on a 4-key sample, and the hoisted schedule with the CUDA-core MAC
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sample_keys = keys[:4]
    o1 = torch.empty_like(cts)
    for k in sample_keys:
        cb.rotate(ctx, k, cts, out=o1)
    torch.cuda.synchronize()
    e0.record(st)
    for k in sample_keys:
        cb.rotate(ctx, k, cts, out=o1)
    e1.record(st)
    torch.cuda.synchronize()
    per_rot = ROT_NCT * len(sample_keys) / (e0.elapsed_time(e1) / 1000.0)
    ctx.tensor_cores = False
    step()
    torch.cuda.synchronize()
    e0.record(st)
    step()
    e1.record(st)
    torch.cuda.synchronize()
    cc_value = rots / (e0.elapsed_time(e1) / 1000.0)
    _, cc_phases = cb.rotate_hoisted_timed(ctx, keys, cts, out=out)
    ctx.tensor_cores = True
    torch.cuda.synchronize()
    plain_gpu = {
        "per_rotation": {"value": per_rot, "unit": "rotations/s", "path": "ckks_rotate (no hoisting, CUDA-core MAC)",
                         "sample": "%d ct x %d keys" % (ROT_NCT, len(sample_keys))},
        "hoisted_cuda_core_mac": {"value": cc_value, "unit": "rotations/s", "path": "ckks_rotate_hoisted, "
                                  "tensor cores off", "mac_ms_per_step": cc_phases["key-switch MAC"]},
    }
    # kernels of one step, counted after every timed region (the tracing hooks stay out of the timing)
    counted = count_launches(step)
    assert ctx.last_mac_path == "tensor_cores", "the headline run must take the tensor-core MAC"
    mac_path = ctx.last_mac_path
    decoded, fresh = rot_decoded_error(cb, ctx, keys, ROT_STEPS, secret, q, n)
    parity, cpu_base = None, None
    if rank == 0 and world == 1:
        # CPU baseline on the GPU arm's own ciphertexts and (downloaded) keys: the
        # oracle's outputs are compared word for word with the GPU's
        threads = os.cpu_count() or 1
        n_cpu = min(threads, ROT_NCT)
        keys_h = [keys[g].download() for g in range(2)]
        v, sample, cpu_out = rot_cpu_sample(n_cpu, 2, keys=keys_h, exps=exps[:2], cts=host)
        gpu_out = cb.to_numpy_u64(out[:n_cpu, :2])
        cpu_base = {"value": v, "unit": "rotations/s", "cores": n_cpu, "kind": "port", "sample": sample}
        od = rot_oracle_decoded(fresh, keys_h[0], exps[0], ROT_STEPS[0], secret, q, p)
        parity = {"words_compared": int(gpu_out.size) + od["words_compared"],
                  "mismatches": int(np.count_nonzero(gpu_out != cpu_out)) + od["mismatches"],
                  "what": "%d ct x 2 keys of the timed batch (tensor-core MAC) and the fresh encryption's key-0 "
                          "rotation, against the oracle's restatement of the reference rotation" % n_cpu}
        decoded["oracle_key0_rel_l2"] = od["key0_rel_l2"]
        decoded["oracle_key0_log2"] = od["key0_log2"]
        decoded["gpu_key0_log2"] = float(np.log2(decoded["key0_rel_l2"])) if decoded["key0_rel_l2"] > 0 else None
    line = {
        "metric": "key-switched rotations/s (N=2^16, 24 limbs, hoisted, bit-exact)", "value": value,
        "unit": "rotations/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts, GPU-generated keys)",
        "config": dict(rot_config(), autotune=tuning.strip().splitlines()),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": mac_traffic, "traffic_source": "one-pass ncu capture of the full-size launch",
                     "peak_kind": kind,
                     "kernel": "k_mac_tc (INT8 tcgen05 key-switch MAC, %d digits, keys %.3f GB each, read once "
                               "per %d ct)" % (D, key_bytes / 1e9, min(group, ROT_NCT)),
                     "kernel_ms_per_step": mac_ms, "algorithmic_bytes_per_step": mac_bytes},
        "whole_rotation_roofline": {"bytes_per_rotation": key_bytes + 2 * ct_bytes,
                                    "frac_no_key_reuse": (key_bytes + 2 * ct_bytes) * value / 1e9 / peak},
        "phases_ms_per_step": phases,
        "decoded_error": decoded,
        "mac_path": mac_path,
        "plain_gpu": plain_gpu,
        "e2e": {"value": rots * e2e_steps * world / e2e_s, "unit": "rotations/s",
                "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(hout.nbytes),
                "path": "ckks_rotate_hoisted_host"},
        # kernels of one step as counted by the profiler hooks (analytic count as the fallback)
        "gpu_launches": args.steps * (counted if counted else groups * (5 * min(group, ROT_NCT) + 5)),
        "clocks": clk,
    }
    if cpu_base:
        line["cpu_baseline"] = cpu_base
        line["parity"] = parity
    return line


def rot_decoded_error(cb, ctx, keys, steps, secret, q, n, seed=77):
    """Decoded error of the rotations against FP64 (numpy) rotations of the
    cleartext, outside every timed region and through the library alone: one
    fresh encryption under the bench's secret (b = m + e - a s, sigma 3.2, scale
    2^50) is rotated by every key, decrypted (b + a s) and decoded on the GPU.
    Returns the largest relative L2 error over the keys and its log2."""
    import torch
    rng = np.random.default_rng(seed)
    L, K = len(q), len(keys)
    x = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    scale = 2.0 ** 50
    m = cb.encode(ctx, x, L, scale)
    a = cb.as_u64_tensor(np.stack([rng.integers(0, qi, n, dtype=np.uint64) for qi in q]))
    e_int = np.rint(rng.normal(0.0, 3.2, n)).astype(np.int64)
    e = cb.as_u64_tensor(np.stack([(e_int % qi).astype(np.uint64) for qi in q]))
    s_res = cb.as_u64_tensor(np.stack([(secret.astype(np.int64) % qi).astype(np.uint64) for qi in q]))
    s_hat = ctx.ntt_forward(s_res.clone())
    a_s = ctx.ntt_inverse(ctx.pointwise(ctx.ntt_forward(a.clone()), s_hat, "mul"))
    b = ctx.pointwise(ctx.pointwise(m, e, "add"), a_s, "sub")
    ct = torch.stack([b, a])[None].contiguous()
    out = cb.rotate_hoisted(ctx, keys, ct)[0]                   # [K][2][L][N]
    s_hat_k = s_hat[None].expand(K, L, n).contiguous()
    a2s = ctx.ntt_inverse(ctx.pointwise(ctx.ntt_forward(out[:, 1].contiguous()), s_hat_k, "mul"))
    dec = cb.decode(ctx, ctx.pointwise(out[:, 0].contiguous(), a2s, "add"), scale).cpu().numpy()
    errs = [float(np.linalg.norm(dec[g] - np.roll(x, -steps[g])) / np.linalg.norm(x)) for g in range(K)]
    worst = max(errs)
    res = {"rel_l2_max": worst, "log2": float(np.log2(worst)) if worst > 0 else None,
           "key0_rel_l2": errs[0],
           "check": "fresh encryption rotated by every key, decoded vs numpy.roll of the FP64 slots"}
    fresh = {"ct": cb.to_numpy_u64(ct[0]), "out0": cb.to_numpy_u64(out[0]), "slots": x, "scale": scale}
    return res, fresh


def rot_oracle_decoded(fresh, key0, exp0, step0, secret, q, p):
    """The oracle's side of the decoded-error check: the same fresh encryption
    rotated by key 0 with the oracle's restatement of the reference rotation,
    compared word for word with the GPU's output and decoded with the oracle's
    FP64 decode (the reference's CkksCanonicalEmbedding order of operations)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    want = o.hybrid_rotate(q, p, key0, exp0, ROT_BASE_LOG, fresh["ct"])
    dec = o.decode(q, o.decrypt(q, secret, want), fresh["scale"])
    x = fresh["slots"]
    err = float(np.linalg.norm(dec - np.roll(x, -step0)) / np.linalg.norm(x))
    return {"key0_rel_l2": err, "key0_log2": float(np.log2(err)) if err > 0 else None,
            "words_compared": int(want.size), "mismatches": int(np.count_nonzero(want != fresh["out0"]))}


def rot_cpu_sample(threads, n_keys=2, keys=None, exps=None, cts=None, n_ct=None):
    """Times the oracle's restatement of the reference's hoisted hybrid-QP
    rotation (hybrid_rns_galois_key.rs:550-780 with bounded_gadget.rs:273-312
    hoisting) on the host: one ciphertext per thread, n_keys Galois keys each,
    each rotation single-threaded (the reference's rayon granularity).
    keys/exps/cts: the GPU arm's own keys (downloaded, reference layout),
    exponents and ciphertexts; generated with the oracle when absent.
    Returns (rotations/s, sample description, outputs [n_ct][n_keys][2][L][N])."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle, P, arr, u64p
    o = Oracle()
    n = 1 << ROT_LOG_N
    n_ct = threads if n_ct is None else n_ct
    q = arr(o.primes_below_bits(ROT_QBITS, n, ROT_L))
    p = arr(o.primes_below_bits(ROT_PBITS, n, ROT_K))
    rng = np.random.default_rng(77)
    if keys is None:
        secret = rng.integers(-1, 2, n).astype(np.int8)
        exps = [int(o.L.oracle_rotation_exponent_left(n, r)) for r in ROT_STEPS[:n_keys]]
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(n_keys) as ex:
            keys = list(ex.map(lambda ik: o.hybrid_key(q, p, secret, ik[1], ROT_BASE_LOG, seed=500 + ik[0]),
                               enumerate(exps)))
    if cts is None:
        cts = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                        for _ in range(n_ct)])
    cts = np.ascontiguousarray(cts[:n_ct])
    keys = [np.ascontiguousarray(k) for k in keys[:n_keys]]
    out = np.zeros((n_ct, n_keys, 2, ROT_L, n), np.uint64)
    kp = (u64p * n_keys)(*[P(k) for k in keys])
    ex_arr = arr(exps[:n_keys])
    t = time.perf_counter()
    o.L.oracle_hybrid_rotate_hoisted_batch(P(q), ROT_L, P(p), ROT_K, n, ROT_BASE_LOG, n_keys, P(ex_arr), kp,
                                           n_ct, P(cts), P(out), threads)
    dt = time.perf_counter() - t
    rots = n_ct * n_keys
    return rots / dt, ("%d ciphertexts x %d Galois keys on %d thread(s) (one ciphertext per thread), N=2^%d, "
                       "%d+%d limbs, base 2^%d: %d rotations in %.2f s"
                       % (n_ct, n_keys, threads, ROT_LOG_N, ROT_L, ROT_K, ROT_BASE_LOG, rots, dt)), out


# ------------------------------------------------- multiply chain (N=2^12)
MUL_LOG_N, MUL_PAIRS, MUL_BASE_LOG = 12, 64, 20
# the reference's prime search at N=2^12: one 60-bit and two 40-bit Q primes, one 60-bit P
MUL_Q = [0xfffffffffffc001, 0xfffffdc001, 0xfffffc6001]
MUL_P = [0xffffffffffe8001]


def mul_config():
    return {"workload": "HMult -> relinearize -> rescale -> rotate by 1 slot, N=2^12, q = 60+40+40 bits, "
                        "P = 60 bits, bounded gadget base 2^20, 64 ciphertext pairs",
            "log_n": MUL_LOG_N, "q_bits": [60, 40, 40], "p_bits": [60], "base_log": MUL_BASE_LOG,
            "pairs": MUL_PAIRS, "scale": "2^40", "secret": "ternary", "sigma": 3.2,
            "l2": "working set (12 MB) fits L2; latency-bound", "parallelism": "replicas"}


def bench_mul_gpu(args, world, rank, local):
    import torch
    import ckks_b200 as cb
    dev = torch.device("cuda", local)
    n = 1 << MUL_LOG_N
    ctx = cb.Context(MUL_LOG_N, MUL_Q, MUL_P)
    tuning = ctx.autotune(limbs=len(MUL_Q) + len(MUL_P), polys=64)  # NTT tile choices, outside the timed region
    rng = np.random.default_rng(99 + rank)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    rk = cb.KeySwitchKey.relin_generate(ctx, 3, MUL_BASE_LOG, secret, seed=5)
    gk = cb.KeySwitchKey.hybrid_generate(ctx, 2, MUL_BASE_LOG, ctx.rotation_exponent_left(1), secret, seed=6)
    hx = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in MUL_Q], axis=1)
                   for _ in range(MUL_PAIRS)])
    hy = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in MUL_Q], axis=1)
                   for _ in range(MUL_PAIRS)])
    x, y = cb.as_u64_tensor(hx, dev), cb.as_u64_tensor(hy, dev)
    prod = torch.empty((MUL_PAIRS, 2, 2, n), dtype=torch.int64, device=dev)
    rot = torch.empty_like(prod)
    st = torch.cuda.current_stream()

    def step(xx, yy):
        cb.multiply_relinearize_rescale(ctx, rk, xx, yy, out=prod)
        cb.rotate(ctx, gk, prod, out=rot)

    for _ in range(args.warmup):
        step(x, y)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        step(x, y)
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    value = MUL_PAIRS * args.steps * world / (ms_max / 1000.0)
    # end to end: pinned host inputs -> device, chain, result -> pinned host
    px = torch.from_numpy(hx.view(np.int64)).pin_memory()
    py = torch.from_numpy(hy.view(np.int64)).pin_memory()
    pout = torch.empty(tuple(rot.shape), dtype=torch.int64).pin_memory()
    dx, dy = torch.empty_like(x), torch.empty_like(y)

    def e2e_step():
        dx.copy_(px, non_blocking=True)
        dy.copy_(py, non_blocking=True)
        step(dx, dy)
        pout.copy_(rot, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    t = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, time.perf_counter() - t)
    # roofline: bytes a chain must move at least (two input ciphertexts, both
    # keys, the output ciphertext) per pair, against the HBM copy peak
    ct_in, ct_out = 2 * 3 * n * 8, 2 * 2 * n * 8
    D_r, w_r = rk.info()
    D_g, w_g = gk.info()
    bytes_step = MUL_PAIRS * (2 * ct_in + ct_out) + 8 * (w_r + w_g)
    peak, kind = peaks()
    achieved = bytes_step / (ms_max / args.steps / 1000.0) / 1e9
    launches = count_launches(lambda: step(x, y))  # after every timed region
    return {
        "metric": "HMult+relinearize+rescale+rotate chains/s (N=2^12, 3 limbs, bit-exact)", "value": value,
        "unit": "chains/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts, GPU-generated keys)",
        "config": dict(mul_config(), autotune=tuning.strip().splitlines()),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": kind,
                     "kernel": "whole chain (working set fits L2: launch/latency-bound)",
                     "algorithmic_bytes_per_step": bytes_step},
        "e2e": {"value": MUL_PAIRS * args.steps * world / e2e_s, "unit": "chains/s",
                "h2d_bytes_per_step": int(hx.nbytes + hy.nbytes), "d2h_bytes_per_step": int(pout.numel() * 8),
                "path": "torch pinned copies + ckks_multiply_relin_rescale + ckks_rotate"},
        "gpu_launches": None if launches is None else args.steps * launches, "clocks": clk,
    }


def mul_cpu_sample(threads, pairs=None):
    """Times the oracle's restatement of the reference chain (tensor, bounded
    relinearize, rescale, hybrid rotate) on the host, one pair per thread."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    import concurrent.futures as cf
    o = Oracle()
    n = 1 << MUL_LOG_N
    pairs = pairs or threads
    rng = np.random.default_rng(7)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    rk = o.relin_key(MUL_Q, secret, MUL_BASE_LOG, seed=5)
    k = int(o.L.oracle_rotation_exponent_left(n, 1))
    gk = o.hybrid_key(MUL_Q[:2], MUL_P, secret, k, MUL_BASE_LOG, seed=6)
    xs = [np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in MUL_Q], axis=1) for _ in range(pairs)]
    ys = [np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in MUL_Q], axis=1) for _ in range(pairs)]

    def chain(i):
        quad = o.tensor(MUL_Q, xs[i], ys[i])
        rel = o.relinearize(MUL_Q, quad, rk, MUL_BASE_LOG)
        resc = o.rescale(MUL_Q, rel.reshape(2, 3, n))
        return o.hybrid_rotate(MUL_Q[:2], MUL_P, gk, k, MUL_BASE_LOG, resc)

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(chain, range(pairs)))
    dt = time.perf_counter() - t
    return pairs / dt, "%d ciphertext pairs over %d threads (one chain per thread), N=2^12, %.2f s" % (
        pairs, threads, dt)


# ------------------------------------------------------ structured CCMM
CCMM_LOG_N, CCMM_L, CCMM_D, CCMM_BASE_LOG = 15, 14, 64, 20


def ccmm_config():
    return {"workload": "structured encrypted CCMM 64x64 by 64x64, one ciphertext per entry, N=2^15, "
                        "14 x 50-bit Q limbs, bounded relinearization base 2^20",
            "log_n": CCMM_LOG_N, "q_limbs": CCMM_L, "d": CCMM_D, "base_log": CCMM_BASE_LOG, "scale": "2^40",
            "l2": "operands (2 x 30 GB) larger than L2", "parallelism": "replicas"}


def ccmm_primes():
    import ckks_b200.params as params
    return params.primes_below_bits(50, 1 << CCMM_LOG_N, CCMM_L)


def bench_ccmm_gpu(args, world, rank, local):
    import torch
    import ckks_b200 as cb
    dev = torch.device("cuda", local)
    n, d, L = 1 << CCMM_LOG_N, CCMM_D, CCMM_L
    q = ccmm_primes()
    ctx = cb.Context(CCMM_LOG_N, q)
    tuning = ctx.autotune(limbs=len(q), polys=64)  # NTT tile choices, outside the timed region
    rng = np.random.default_rng(31 + rank)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    rk = cb.KeySwitchKey.relin_generate(ctx, L, CCMM_BASE_LOG, secret, seed=9)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    A = torch.empty((d * d, 2, L, n), dtype=torch.int64, device=dev)
    B = torch.empty_like(A)
    for l, m in enumerate(q):  # uniform residues per limb (fresh-ciphertext distribution)
        A[:, :, l].random_(0, m, generator=gen)
        B[:, :, l].random_(0, m, generator=gen)
    C = torch.empty((d * d, 2, L - 1, n), dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream()

    def step():
        cb.matmul_structured(ctx, rk, A, B, d, d, d, out=C)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        step()
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    value = args.steps * world / (ms_max / 1000.0)
    D, key_words = rk.info()
    ct_bytes = 2 * L * n * 8
    # algorithmic bytes: both operand matrices read, the product written, and
    # the relinearization key read once per group of four outputs
    bytes_step = 2 * d * d * ct_bytes + d * d * 2 * (L - 1) * n * 8 + (d * d // 4) * key_words * 8
    peak, kind = peaks()
    achieved = bytes_step / (ms_max / args.steps / 1000.0) / 1e9
    # end to end: pinned host operands in, product out, through the same call
    hA = torch.empty(tuple(A.shape), dtype=torch.int64).pin_memory()
    hB = torch.empty(tuple(B.shape), dtype=torch.int64).pin_memory()
    hC = torch.empty(tuple(C.shape), dtype=torch.int64).pin_memory()
    hA.copy_(A)
    hB.copy_(B)
    torch.cuda.synchronize()
    barrier(world)
    t = time.perf_counter()
    A.copy_(hA, non_blocking=True)
    B.copy_(hB, non_blocking=True)
    step()
    hC.copy_(C, non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, time.perf_counter() - t)
    launches_per_step = count_launches(step)  # after every timed region
    parity = ccmm_parity(cb, ctx, rk, A, B, C, q) if (rank == 0 and world == 1) else None
    return {
        "metric": "64x64 structured CCMM/s (N=2^15, 14 limbs, both operands encrypted, bit-exact)", "value": value,
        "unit": "CCMM/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded uniform ciphertext residues, GPU-generated key)",
        "config": dict(ccmm_config(), autotune=tuning.strip().splitlines()),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": kind, "kernel": "whole CCMM (operands, product, key stream)",
                     "algorithmic_bytes_per_step": bytes_step},
        "e2e": {"value": world / e2e_s, "unit": "CCMM/s", "h2d_bytes_per_step": int(2 * A.numel() * 8),
                "d2h_bytes_per_step": int(C.numel() * 8), "path": "torch pinned copies + ckks_ccmm_structured"},
        "gpu_launches": None if launches_per_step is None else args.steps * launches_per_step, "clocks": clk,
        "parity": parity,
    }


def ccmm_parity(cb, ctx, rk, A, B, C, q):
    """Output entry (0, 0) of the timed product recomputed by the oracle from
    the same operands and key: 64 tensors summed, bounded relinearization,
    rescale (matrix/rns_ckks_ciphertext.rs:220-318), compared word for word."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    n, d, L = 1 << CCMM_LOG_N, CCMM_D, CCMM_L
    row = cb.to_numpy_u64(A[0::d])             # A[0 + k d], k = 0..d-1 (column-major)
    col = cb.to_numpy_u64(B[0:d])              # B[k + 0 d]
    key_ntt = rk.download().reshape(-1, L, n)
    key = o.ntt_inverse(q, key_ntt).reshape(-1, 2, L, n)  # the reference's coefficient-domain layout
    acc = None
    for kk in range(d):
        t = o.tensor(q, row[kk], col[kk]).astype(object)
        acc = t if acc is None else acc + t
    quad = np.stack([acc[:, l] % q[l] for l in range(L)], axis=1).astype(np.uint64)
    want = o.rescale(q, o.relinearize(q, quad, key, CCMM_BASE_LOG).reshape(2, L, n))
    got = cb.to_numpy_u64(C[0])
    return {"words_compared": int(want.size), "mismatches": int(np.count_nonzero(got != want)),
            "what": "output entry (0, 0): 64 tensors + relinearization + rescale, against the oracle's "
                    "restatement of the reference"}


def ccmm_object(args, world, rank, local):
    """The 64x64 CCMM measured beside the headline rotations (same run): 3
    timed products after 3 warm-up ones, with its own roofline, e2e, parity
    and, at N=1, the CPU baseline."""
    import copy
    a = copy.copy(args)
    a.steps, a.warmup = 3, 3
    line = bench_ccmm_gpu(a, world, rank, local)
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        v, sample = ccmm_cpu_sample(threads)
        line["cpu_baseline"] = {"value": v, "unit": "CCMM/s", "cores": threads, "kind": "port", "sample": sample}
    keep = ["metric", "value", "unit", "steps", "warmup", "ms_per_step", "higher_is_better", "config", "roofline",
            "e2e", "gpu_launches", "clocks", "parity", "cpu_baseline"]
    return {k: line[k] for k in keep if k in line}


def park_object(args, world, rank, local):
    """Park Mod-PP-MM at n = 4096 measured beside the headline rotations (same
    run): 5 timed products after 3 warm-up ones, with its own roofline, e2e,
    parity, the CUDA-core form and, at N=1, the CPU baseline."""
    import copy
    a = copy.copy(args)
    a.steps, a.warmup = 5, 3
    line = bench_park_gpu(a, world, rank, local)
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        v, sample = park_cpu_sample(threads, a.park_n)
        line["cpu_baseline"] = {"value": v, "unit": "products/s", "cores": threads, "kind": "port", "sample": sample}
    keep = ["metric", "value", "unit", "steps", "warmup", "ms_per_step", "higher_is_better", "config", "roofline",
            "plain_gpu", "e2e", "gpu_launches", "clocks", "parity", "cpu_baseline"]
    return {k: line[k] for k in keep if k in line}


def ccmm_cpu_sample(threads):
    """Times the oracle's restatement of one output entry of the reference
    CCMM (64 tensors summed, bounded relinearization, rescale) per thread at
    N=2^15, 14 limbs; CCMM/s = threads / (4096 x entry time)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    import concurrent.futures as cf
    o = Oracle()
    n, d, L = 1 << CCMM_LOG_N, CCMM_D, CCMM_L
    q = [int(x) for x in o.primes_below_bits(50, n, L)]
    rng = np.random.default_rng(5)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    key = o.relin_key(q, secret, CCMM_BASE_LOG, seed=9)
    row = [np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1) for _ in range(d)]
    col = [np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1) for _ in range(d)]

    def entry(_):
        acc = None
        for kk in range(d):
            t = o.tensor(q, row[kk], col[kk])
            acc = t if acc is None else np.stack([(acc[:, l] + t[:, l]) % q[l] for l in range(L)], axis=1)
        rel = o.relinearize(q, acc, key, CCMM_BASE_LOG)
        return o.rescale(q, rel.reshape(2, L, n))

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(entry, range(threads)))
    dt = time.perf_counter() - t
    return threads / (d * d * dt), ("%d output entries (64 tensors + relinearize + rescale each, one per thread), "
                                    "N=2^15, 14 limbs, %.1f s" % (threads, dt))


# -------------------------------------------------------------- FFT2 (images)
FFT2_LOG_N, FFT2_S, FFT2_L, FFT2_K, FFT2_IMAGES, FFT2_BASE_LOG = 16, 256, 24, 3, 8, 32


def fft2_config():
    return {"workload": "encrypted 2-D FFT of 256x256 real images, 2 ciphertexts per image at N=2^16, "
                        "24 x 50-bit Q + 3 x 60-bit P, radix-4 diagonal-rotation schedule (4 row + 4 column "
                        "stages, 6 rotations + 7 plaintext products per stage), 8 images per step",
            "log_n": FFT2_LOG_N, "image": [FFT2_S, FFT2_S], "images": FFT2_IMAGES, "q_limbs": FFT2_L,
            "p_limbs": FFT2_K, "base_log": FFT2_BASE_LOG, "scale": "2^50",
            "l2": "keys (about 35 GB) larger than L2", "parallelism": "replicas"}


def bench_fft2_gpu(args, world, rank, local):
    import torch
    import ckks_b200 as cb
    import ckks_b200.params as params
    from ckks_b200 import fft2
    dev = torch.device("cuda", local)
    n = 1 << FFT2_LOG_N
    q = params.primes_below_bits(50, n, FFT2_L)
    p = params.primes_below_bits(60, n, FFT2_K)
    ctx = cb.Context(FFT2_LOG_N, q, p)
    tuning = ctx.autotune(limbs=len(q) + len(p), polys=64)  # NTT tile choices, outside the timed region
    rng = np.random.default_rng(55 + rank)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    plan = fft2.Fft2Plan(ctx, FFT2_S, FFT2_L, secret, base_log=FFT2_BASE_LOG)
    key_bytes = sum(8 * k.info()[1] for st in plan.stages for k in st[2])
    host = np.stack([np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                               for _ in range(2)]) for _ in range(FFT2_IMAGES)])
    cts = cb.as_u64_tensor(host, dev)
    st = torch.cuda.current_stream()

    def step(x):
        return plan.apply(x)

    for _ in range(args.warmup):
        step(cts)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        out = step(cts)
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    value = FFT2_IMAGES * args.steps * world / (ms_max / 1000.0)
    rotations = sum(len(st_[2]) for st_ in plan.stages[:-1]) * 2 * FFT2_IMAGES + 2 * FFT2_IMAGES
    # algorithmic bytes: every key once per stage batch, ciphertexts in and out of every stage
    ct_bytes = lambda lvl: 2 * lvl * n * 8
    lv = [st_[1] for st_ in plan.stages]
    bytes_step = key_bytes + sum(2 * FFT2_IMAGES * (ct_bytes(l) + ct_bytes(l - 1)) for l in lv)
    peak, kind = peaks()
    achieved = bytes_step / (ms_max / args.steps / 1000.0) / 1e9
    pin_in = torch.from_numpy(host.view(np.int64)).pin_memory()
    pin_out = torch.empty(tuple(out.shape), dtype=torch.int64).pin_memory()
    d_in = torch.empty_like(cts)
    torch.cuda.synchronize()
    barrier(world)
    t = time.perf_counter()
    d_in.copy_(pin_in, non_blocking=True)
    o2 = step(d_in)
    pin_out.copy_(o2, non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(world, time.perf_counter() - t)
    launches_per_step = count_launches(lambda: step(cts))  # after every timed region
    return {
        "metric": "encrypted 256x256 FFT2 images/s (N=2^16, 24 limbs, radix-4 schedule, bit-exact)",
        "value": value, "unit": "images/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded uniform ciphertexts, GPU-generated keys, GPU-encoded diagonals)",
        "config": dict(fft2_config(), autotune=tuning.strip().splitlines()),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": kind,
                     "kernel": "whole FFT2 (key streams and stage ciphertexts; rotations per step: %d)" % rotations,
                     "algorithmic_bytes_per_step": bytes_step},
        "e2e": {"value": FFT2_IMAGES * world / e2e_s, "unit": "images/s", "h2d_bytes_per_step": int(host.nbytes),
                "d2h_bytes_per_step": int(pin_out.numel() * 8), "path": "torch pinned copies + ckks_fft_stage(_multi)"},
        "gpu_launches": None if launches_per_step is None else args.steps * launches_per_step, "clocks": clk,
    }


def fft2_cpu_sample(threads):
    """Times the oracle's restatement of one radix-4 row stage (6 hoisted
    rotations, 7 plaintext products, sum, rescale) on one ciphertext per
    thread at level 20 (the middle of the 24 .. 17 levels the 8 stages use);
    images/s = threads / (16 x stage time)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle, P, arr, u64p
    import concurrent.futures as cf
    o = Oracle()
    n, lvl = 1 << FFT2_LOG_N, 20
    q = arr(o.primes_below_bits(50, n, FFT2_L))[:lvl]
    p = arr(o.primes_below_bits(60, n, FFT2_K))
    rng = np.random.default_rng(3)
    secret = rng.integers(-1, 2, n).astype(np.int8)
    offs = [-3, -2, -1, 1, 2, 3]
    exps = [int(o.L.oracle_rotation_exponent_left(n, x)) if x > 0 else int(o.L.oracle_rotation_exponent_right(n, -x))
            for x in offs]
    with cf.ThreadPoolExecutor(6) as ex:
        keys = list(ex.map(lambda ie: o.hybrid_key(q, p, secret, ie[1], FFT2_BASE_LOG, seed=900 + ie[0]),
                           enumerate(exps)))
    plains = [np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(7)]
    cts = np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                    for _ in range(threads)])
    rot = np.zeros((threads, 6, 2, lvl, n), np.uint64)
    kp = (u64p * 6)(*[P(k) for k in keys])
    ex_arr = arr(exps)

    def finish(c):
        acc = o.mul_plain(q, cts[c], plains[6]).astype(object)
        for g in range(6):
            acc = acc + o.mul_plain(q, rot[c, g], plains[g]).astype(object)
        acc = np.stack([acc[:, l] % int(q[l]) for l in range(lvl)], axis=1).astype(np.uint64)
        return o.rescale(q, acc)

    t = time.perf_counter()
    o.L.oracle_hybrid_rotate_hoisted_batch(P(q), lvl, P(p), FFT2_K, n, FFT2_BASE_LOG, 6, P(ex_arr), kp, threads,
                                           P(cts), P(rot), threads)
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(finish, range(threads)))
    dt = time.perf_counter() - t
    return threads / (16 * dt), ("%d ciphertexts x one radix-4 stage at level 20 (6 hoisted rotations, 7 plaintext "
                                 "products, rescale; one ciphertext per thread), %.1f s; x16 stage-ciphertexts "
                                 "per image" % (threads, dt))


def free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_replicas(args):
    """`--gpus N` without a torchrun environment: re-executes this command as
    N ranks (one process per GPU) under torch.distributed.run on 127.0.0.1.
    The b200 arm needs N visible GPUs and stops with an error otherwise; the
    reference arm runs on the host cores (rank 0 measures, the others exit)."""
    if args.impl == "b200":
        import torch
        have = torch.cuda.device_count()
        if have < args.gpus:
            raise SystemExit("bench.py: --gpus %d but only %d CUDA device(s) are visible" % (args.gpus, have))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % args.gpus,
           "--master-addr=127.0.0.1", "--master-port=%d" % free_port(), os.path.abspath(__file__)] + sys.argv[1:]
    sys.stdout.flush()
    os.execv(sys.executable, cmd)


PARK_N = 4096
PARK_Q = 0x7ffff6001  # research_profile_4096's first modulus, the reference characterization's


def bench_park_gpu(args, world, rank, local):
    """Park Mod-PP-MM (ccmm/park.rs:1634-1647) at n = 4096 (the reference's
    characterization sizes run 256 .. 4096, src/bin/park_mod_pp_mm_characterization.rs):
    square u64 matrices of residues, exact (lhs x rhs) mod q per step."""
    import torch
    import ckks_b200 as cb
    dev = torch.device("cuda", local)
    n, q = args.park_n, PARK_Q
    gen = torch.Generator(device=dev)
    gen.manual_seed(77 + rank)
    A = torch.empty((n, n), dtype=torch.int64, device=dev).random_(0, q, generator=gen)
    B = torch.empty((n, n), dtype=torch.int64, device=dev).random_(0, q, generator=gen)
    C = torch.empty((n, n), dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream()

    gemm_ms = []

    def step(backend="tensor_cores"):
        cb.park_mod_pp_mm(A, B, q, out=C, backend=backend)
        if backend == "tensor_cores":
            gemm_ms.append(cb.park_last_timing()[1])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    gemm_ms.clear()
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        step()
    t1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    clk = clocks.stop()
    ms_max = max_over_ranks(world, ms)
    value = args.steps * world / (ms_max / 1000.0)
    gemm = sum(gemm_ms) / len(gemm_ms)
    # the plain GPU form: the same product with 192-bit sums on the CUDA cores
    C2 = torch.empty_like(C)
    cb.park_mod_pp_mm(A, B, q, out=C2, backend="cuda_cores")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    cb.park_mod_pp_mm(A, B, q, out=C2, backend="cuda_cores")
    e1.record(st)
    torch.cuda.synchronize()
    cuda_core_ms = e0.elapsed_time(e1)
    backends_equal = bool(torch.equal(C, C2))
    del C2
    # parity of sampled outputs against the oracle (outside the timed region)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    a, b, c = cb.to_numpy_u64(A), cb.to_numpy_u64(B), cb.to_numpy_u64(C)
    rows = [0, (7 * n) // 16, n - 1]
    mism = sum(int(np.count_nonzero(o.park_mod_pp_mm(a[r:r + 1], b, q) != c[r:r + 1])) for r in rows)
    # end to end: each step copies both operands from pinned host memory, runs the
    # product through the public call and reads the result back (CUDA events)
    Ah, Bh = A.cpu().pin_memory(), B.cpu().pin_memory()
    Ch = torch.empty_like(Ah).pin_memory()

    def e2e_step():
        A.copy_(Ah, non_blocking=True)
        B.copy_(Bh, non_blocking=True)
        cb.park_mod_pp_mm(A, B, q, out=C)
        Ch.copy_(C, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(args.steps):
        e2e_step()
    e1.record(st)
    torch.cuda.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1000.0 / args.steps
    e2e_equal = bool(torch.equal(Ch, C.cpu()))
    # the dominant kernel k_park_tc runs nb^2 n^3 unsigned 8-bit multiply-adds (nb = 5 bytes
    # per residue of the 35-bit modulus) on the tensor cores; INT8 dense is twice the bf16
    # dense rate on B200, so the peak is twice the measured bf16 burst figure
    nb = ((q - 1).bit_length() + 7) // 8
    ops = 2.0 * nb * nb * float(n) ** 3
    bf16, bf16_kind = bf16_peak()
    i8_peak = 2.0 * bf16 if bf16 else None
    achieved = ops / (gemm / 1000.0) / 1e12
    return {"metric": park_metric(n), "value": value,
            "unit": "products/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform residues)",
            "config": park_config(n),
            "roofline": {"bound": "tensor", "achieved": achieved, "unit": "TOP/s (INT8)", "peak": i8_peak,
                         "frac": achieved / i8_peak if i8_peak else None,
                         # DRAM bytes of one launch at n = 2048 (read 127.0 MB, write 23.4 MB: the
                         # packed operands once and the product), scaled by n^2 like those arrays
                         "traffic": (127.0e6 + 23.4e6) * (n / 2048.0) ** 2,
                         "traffic_source": "ncu capture of the n=2048 launch, scaled by (n/2048)^2",
                         "kernel": "k_park_tc (INT8 tcgen05 products of byte planes, %d x %d planes)" % (nb, nb),
                         "kernel_ms": gemm, "rest_of_step_ms": (ms_max / args.steps) - gemm,
                         "peak_source": "2 x bf16 dense (%s %s)" % (bf16_kind, bf16),
                         "ops_per_launch": ops},
            "plain_gpu": {"backend": "cuda_cores (k_park_mm, 192-bit exact sums)", "ms": cuda_core_ms,
                          "value": 1000.0 / cuda_core_ms, "unit": "products/s", "words_equal": backends_equal},
            "e2e": {"value": 1.0 / e2e_s, "unit": "products/s", "h2d_bytes_per_step": 2 * n * n * 8,
                    "d2h_bytes_per_step": n * n * 8, "result_equal": e2e_equal,
                    "path": "pinned host operands -> park_mod_pp_mm (tensor cores) -> pinned host result"},
            "parity": {"words_compared": len(rows) * n, "mismatches": mism,
                       "what": "three full output rows against the oracle's Reference backend"},
            "gpu_launches": 3 * args.steps, "clocks": clk}


def park_metric(n):
    return "Park Mod-PP-MM/s (n=%d square, modulus 0x7ffff6001, bit-exact)" % n


def park_config(n):
    return {"workload": "Park Mod-PP-MM, %d x %d by %d x %d, u64 residues mod 0x7ffff6001" % (n, n, n, n),
            "n": n, "modulus": PARK_Q, "l2": "operands %d MB each%s" % (
                n * n * 8 // 10**6, ", above L2" if n * n * 8 > 126 * 10**6 else "")}


def park_cpu_sample(threads, n=PARK_N):
    """The oracle's Reference backend (u128 accumulator reduced every term) on an
    n = 512 product, one row block per thread; scaled to n = 4096 by n^3."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    import concurrent.futures as cf
    o = Oracle()
    m = 512
    rng = np.random.default_rng(3)
    a = rng.integers(0, PARK_Q, (m, m), dtype=np.uint64)
    b = rng.integers(0, PARK_Q, (m, m), dtype=np.uint64)
    blocks = np.array_split(np.arange(m), threads)
    t = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda r: o.park_mod_pp_mm(np.ascontiguousarray(a[r]), b, PARK_Q), blocks))
    dt = time.perf_counter() - t
    scale = (m / n) ** 3
    return scale / dt, "one 512 x 512 product over %d threads in %.2f s, scaled by (512/%d)^3" % (threads, dt, n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="rotation", choices=["rotation", "ntt", "multiply", "ccmm", "fft2", "park"])
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    # rotation workload sizes (defaults: the headline configuration; smaller
    # values only for profiling captures that must stay within a few GB)
    ap.add_argument("--rot-limbs", type=int, default=24)
    ap.add_argument("--rot-ct", type=int, default=16)
    ap.add_argument("--rot-keys", type=int, default=32)
    ap.add_argument("--rot-base-log", type=int, default=32)
    ap.add_argument("--rot-log-n", type=int, default=16)
    # Park product size (default: the characterization's largest, n = 4096)
    ap.add_argument("--park-n", type=int, default=PARK_N)
    ap.add_argument("--no-ccmm", action="store_true",
                    help="rotation workload: leave out the 64x64 CCMM measured beside it")
    ap.add_argument("--no-park", action="store_true",
                    help="rotation workload: leave out the Park Mod-PP-MM measured beside it")
    args = ap.parse_args()
    if args.gpus < 1:
        ap.error("--gpus must be at least 1")
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        launch_replicas(args)  # does not return
    if int(os.environ.get("WORLD_SIZE", "1")) != args.gpus:
        raise SystemExit("bench.py: --gpus %d but WORLD_SIZE=%s" % (args.gpus, os.environ.get("WORLD_SIZE")))
    global ROT_L, ROT_NCT, ROT_STEPS, ROT_BASE_LOG, ROT_LOG_N
    ROT_L, ROT_NCT, ROT_BASE_LOG, ROT_LOG_N = args.rot_limbs, args.rot_ct, args.rot_base_log, args.rot_log_n
    ROT_STEPS = ROT_STEPS[:args.rot_keys]
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup() if args.impl == "b200" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        line = reference_arm(args, world, rank)
        if line:
            print(json.dumps(line), flush=True)
        return
    if args.workload == "fft2":
        line = bench_fft2_gpu(args, world, rank, local)
        if rank == 0 and world == 1:
            threads = os.cpu_count() or 1
            v, sample = fft2_cpu_sample(threads)
            line["cpu_baseline"] = {"value": v, "unit": "images/s", "cores": threads, "kind": "port",
                                    "sample": sample}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "park":
        line = bench_park_gpu(args, world, rank, local)
        if rank == 0 and world == 1:
            threads = os.cpu_count() or 1
            v, sample = park_cpu_sample(threads, args.park_n)
            line["cpu_baseline"] = {"value": v, "unit": "products/s", "cores": threads, "kind": "port",
                                    "sample": sample}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "ccmm":
        line = bench_ccmm_gpu(args, world, rank, local)
        if rank == 0 and world == 1:
            threads = os.cpu_count() or 1
            v, sample = ccmm_cpu_sample(threads)
            line["cpu_baseline"] = {"value": v, "unit": "CCMM/s", "cores": threads, "kind": "port", "sample": sample}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "multiply":
        line = bench_mul_gpu(args, world, rank, local)
        if rank == 0 and world == 1:
            threads = os.cpu_count() or 1
            v, sample = mul_cpu_sample(threads, pairs=4 * threads)
            line["cpu_baseline"] = {"value": v, "unit": "chains/s", "cores": threads, "kind": "port",
                                    "sample": sample}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "ntt":
        line = bench_ntt_gpu(args, world, rank, local)
    else:
        line = bench_rot_gpu(args, world, rank, local)
        if not args.no_ccmm:
            # the metric's second half: one 64x64 CCMM at the CCMM configuration,
            # measured in the same run after the rotation's memory is released
            import gc
            import torch
            gc.collect()
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            line["ccmm"] = ccmm_object(args, world, rank, local)
        if not args.no_park:
            import gc
            import torch
            gc.collect()
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            line["park"] = park_object(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        v, sample = ntt_cpu_sample(threads, seconds_target=10.0)
        line["cpu_baseline"] = {"value": v, "unit": "limb-NTT/s", "cores": threads, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
