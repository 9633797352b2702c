"""RS(32,32) encode throughput on B200 (the reference's headline shape).

Workload: GF(2^8) ReedSolomon(32, 32) encode, 1 MiB shards of uniform random bytes
(seeded, generated on the device), STRIPES stripes per step, all resident in HBM. A
step is one batched launch over all stripes (the FFT route, bitsliced). Inputs (32 GiB
of data per step at the default size) are far larger than L2, so no flush is needed.

Metric: algorithmic GB/s = (k + m) * shard_bytes * stripes / step time (read k shards,
write m parity shards per stripe), also as a fraction of measured HBM copy bandwidth.
Alongside: the plain matrix kernel one stripe per launch, the end-to-end rate through
the public host-pointer API from pinned host memory, and the CPU baseline (the oracle's
multi-threaded restatement of the reference's GFNI FFT path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Other workloads (one JSON line each, 1 GPU, no reference arm):
    --workload stripes   RS(32,32) and RS(16,16) encode (FFT and matrix routes) and
                         reconstruct, 4 KiB / 64 KiB / 1 MiB shards, 4096 stripes
    --workload mixed     10,000 stripes of nine shapes, 25% reconstruct: batched+tuned
                         (graph) against one plain launch per stripe
    --workload rs16      ReedSolomon16 (1024,1024) and (4096,12288), 2 KiB shards
    --workload serve     Poisson request stream at 50k req/s through the request server
    --workload tuner     exhaustive autotuning of sampled workloads, the MLP cost model
                         trained on them, held-out regret (model and default)
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

K_DATA, M_PARITY = 32, 32
SHARD = 1 << 20
METRIC = "RS(32,32) encode GB/s & % HBM peak, batched+tuned vs plain, 1 B200 bit-exact"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--stripes", type=int, default=1024, help="stripes per step per GPU")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the untimed-region extras (reconstruct and mixed-batch figures)")
    ap.add_argument("--workload", default="encode",
                    choices=["encode", "stripes", "mixed", "rs16", "serve", "tuner"])
    ap.add_argument("--save-model", default=None,
                    help="tuner workload: write the trained cost model here and its timings beside it (.npz)")
    ap.add_argument("--tuner-workloads", type=int, default=10000,
                    help="workloads the tuner times (about 5 applicable configurations each)")
    ap.add_argument("--requests", type=int, default=400, help="requests of the serve workload")
    ap.add_argument("--rs16", default=None,
                    help="rs16 workload: shapes K,M,STRIPES[,SHARD_BYTES] separated by '/' instead of both")
    ap.add_argument("--mixed-stripes", type=int, default=10000, help="stripes of the mixed workload")
    ap.add_argument("--mixed-packed", action="store_true",
                    help="mixed workload: rows packed back to back at their (odd) lengths")
    ap.add_argument("--stripes-shapes", default=None,
                    help="stripes workload: shapes K,M separated by '/' (default 32,32/16,16)")
    ap.add_argument("--stripes-sizes", default=None,
                    help="stripes workload: shard bytes separated by ',' (default 4096,65536,1048576)")
    ap.add_argument("--stripes-count", type=int, default=4096, help="stripes workload: stripes per launch")
    return ap.parse_args()


def rank_seed(rank):
    """Each replica encodes its own stripes (weak scaling: no data is shared)."""
    return 1234 + rank


def max_over_ranks(ms, dist, device):
    """The job's time: the slowest rank's (all ranks take part, then meet at a barrier)."""
    if not dist:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def job_gbs(bytes_per_rank_step, world, ms_per_step):
    """Whole-job algorithmic GB/s: every rank's bytes over the max-over-ranks step time."""
    return bytes_per_rank_step * world / (ms_per_step * 1e-3) / 1e9


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the FFT kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "fft_kk_kernel_32_rs32x32_1MiB.md")
    if not os.path.exists(path):
        return None, None
    per_stripe = None
    for line in open(path):
        if line.startswith("dram_bytes_per_stripe:"):
            per_stripe = float(line.split(":")[1])
    return per_stripe, os.path.relpath(path, ROOT)


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.samples = []
        if self.proc is None:
            return
        time.sleep(0.2)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.samples.append(f)

    def summary(self):
        if not self.samples:
            return None
        sm = [float(f[1]) for f in self.samples if f[1].replace(".", "").isdigit()]
        mx = [float(f[2]) for f in self.samples if f[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for f in self.samples for i in range(4) if f[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def host_cpu():
    """The host CPU as the baseline ran on it: model string, usable threads, ISA flags."""
    model, flags = "unknown", set()
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name") and model == "unknown":
                model = line.split(":", 1)[1].strip()
            elif line.startswith("flags") and not flags:
                flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    usable = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"model": model, "nproc": usable, "logical_cpus": os.cpu_count(),
            "isa": [f for f in ("gfni", "avx512f", "avx512bw", "avx2") if f in flags]}


def _check_cpu_parity(O, stripes, k, m):
    """Byte-check the timed encoder's output against the oracle's scalar encode at
    4096 sampled columns of the first and last stripe (encoding is column-wise)."""
    rng = np.random.default_rng(11)
    L = stripes.shape[2]
    cols = np.sort(rng.choice(L, size=min(L, 4096), replace=False))
    for s in (0, stripes.shape[0] - 1):
        sub = np.ascontiguousarray(stripes[s][:, cols])
        if not np.array_equal(sub[k:], O.encode8(k, m, sub[:k])):
            raise RuntimeError("CPU baseline parity differs from the oracle (stripe %d)" % s)


def cpu_baseline(seconds, threads=None, details=True):
    """The oracle's restatement of the reference's x86 encode (straight-line GFNI/AVX-512
    code generated from the LCH program, as the reference's macro-expanded zmm cores),
    one stripe per thread on all usable host threads, looped over a bounded sample for
    about `seconds`; byte-checked against the oracle after timing. Also one thread on
    one cache-resident 10 KB stripe and one 1 MiB stripe, the sizes the reference
    publishes for RS(32,32) (32,404 and 14,665 MiB/s payload on one Zen 5 core)."""
    from oracle import oracle as O

    k, m = K_DATA, M_PARITY
    cpu = host_cpu()
    threads = threads or cpu["nproc"]
    n_stripes = max(threads, 16)
    shard = SHARD
    rng = np.random.default_rng(7)
    stripes = rng.integers(0, 256, size=(n_stripes, k + m, shard), dtype=np.uint8)
    total_t, total_b, reps = 0.0, 0, 0
    while total_t < seconds:
        total_t += O.encode8_batch_mt(k, m, stripes, threads)
        total_b += n_stripes * (k + m) * shard
        reps += 1
    _check_cpu_parity(O, stripes, k, m)
    single = {}
    for label, L, budget in (("10KB", 10240, 1.0), ("1MiB", SHARD, 2.0)) if details else ():
        one = rng.integers(0, 256, size=(k + m, L), dtype=np.uint8)
        t1 = O.encode8_repeat(k, m, one, 1)
        n = max(1, int(budget / max(t1, 1e-6)))
        t = O.encode8_repeat(k, m, one, n)
        single[label] = {"payload_mib_s": n * k * L / t / 2**20, "algorithmic_gbs": n * (k + m) * L / t / 1e9,
                         "passes": n}
    sample = ("%d stripes x RS(32,32) x 1 MiB shards, %d passes (%.1f s), one stripe per thread on %d threads, "
              "%s path; byte-checked against the oracle" % (n_stripes, reps, total_t, threads,
                                                            O.cpu_path(k, m, shard)))
    return {"value": total_b / total_t / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": sample, "cpu": cpu, "single_thread": single,
            "published_single_thread_payload_mib_s": {"10KB": 32404, "1MiB": 14665,
                                                      "host": "AMD Zen 5 (GCP c4d), 1 thread"}}


def run_reference(args, rank):
    if rank != 0:
        return
    steps = []
    base = cpu_baseline(1.0)  # untimed: host details, single-thread rates, byte check
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(max(1.0, args.cpu_seconds / max(args.steps, 1)), details=False)
        if i >= args.warmup:
            steps.append(b["value"])
            base["sample"] = b["sample"]
    value = statistics.mean(steps)
    # A step is our arm's step (args.stripes stripes of 1 MiB shards); the CPU time for it
    # is extrapolated from the bounded sample's rate.
    step_bytes = args.stripes * (K_DATA + M_PARITY) * SHARD
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_bytes / (value * 1e9) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform bytes)",
        "config": {"workload": "RS(32,32) encode, 1 MiB shards, %d stripes per launch" % args.stripes,
                   "k": K_DATA, "m": M_PARITY, "shard_bytes": SHARD, "stripes_per_step": args.stripes},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": base["cores"], "kind": "port",
                         "sample": base["sample"], "cpu": base["cpu"], "single_thread": base["single_thread"],
                         "published_single_thread_payload_mib_s": base["published_single_thread_payload_mib_s"]},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def device_parity_prefix(rs, shards, k, length):
    """The first 64 parity bytes of row 0 recomputed by the device-resident batched encode
    (a self-check of the host-pointer path, outside any timed region)."""
    import torch

    d = torch.from_numpy(np.stack([s[:64] for s in shards[:k]])).cuda()
    p = torch.empty((1, rs.parity_shard_count(), 64), dtype=torch.uint8, device="cuda")
    rs.encode_batch_dev(d[None], p, 64, 1)
    torch.cuda.synchronize()
    return p[0, 0].cpu().numpy()


def run_ours(args, rank, world):
    import torch

    import __graft_entry__

    rsb = __graft_entry__.load_package()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist

    S, L, k, m = args.stripes, SHARD, K_DATA, M_PARITY
    g = torch.Generator(device="cuda").manual_seed(rank_seed(rank))
    data = torch.randint(0, 256, (S, k, L), dtype=torch.uint8, device="cuda", generator=g)
    parity = torch.empty((S, m, L), dtype=torch.uint8, device="cuda")
    rs = rsb.ReedSolomon(k, m)
    stream = torch.cuda.current_stream().cuda_stream
    bytes_per_step = S * (k + m) * L

    def step():
        rs.encode_batch_dev(data, parity, L, S, stream=stream)

    # Self-check before timing: matrix-route verify of FFT-route parity on two stripes.
    step()
    torch.cuda.synchronize()
    for s in (0, S - 1):
        shards = [data[s, i] for i in range(k)] + [parity[s, j] for j in range(m)]
        if not rs.verify_dev(shards, L, stream=stream):
            raise RuntimeError("self-check failed: parity of stripe %d does not verify" % s)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = rsb.kernel_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(dev) as clk:
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for i in range(args.steps):
            ev[i][0].record()
            step()
            ev[i][1].record()
        t1.record()
        torch.cuda.synchronize()
    launches = rsb.kernel_launch_count() - launches0
    total_ms = t0.elapsed_time(t1)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(total_ms, dist, "cuda")
    ms_per_step = total_ms / args.steps
    value = job_gbs(bytes_per_step, world, ms_per_step)

    # Plain: the matrix kernel, one stripe per launch.
    rs_plain = rsb.ReedSolomon(k, m)
    rs_plain.set_route("matrix")
    n_plain = min(S, 16)
    for s in range(2):
        rs_plain.encode_batch_dev(data[s], parity[s], L, 1, stream=stream)
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record()
    for s in range(n_plain):
        rs_plain.encode_batch_dev(data[s], parity[s], L, 1, stream=stream)
    p1.record()
    torch.cuda.synchronize()
    plain_gbs = n_plain * (k + m) * L / (p0.elapsed_time(p1) * 1e-3) / 1e9

    # End to end through the host-pointer API from pinned memory: H2D data, encode,
    # D2H parity inside the timed region.
    S_e2e = min(S, 64)
    h_data = torch.empty((S_e2e, k, L), dtype=torch.uint8, pin_memory=True)
    h_par = torch.empty((S_e2e, m, L), dtype=torch.uint8, pin_memory=True)
    h_data.copy_(data[:S_e2e].cpu())
    e2e_times = []
    for rep in range(3):
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        rs.encode_batch_host(h_data.numpy(), h_par.numpy(), L, S_e2e)
        e2e_times.append(time.perf_counter() - t_start)
    e2e_t = min(e2e_times[1:])
    e2e_gbs = S_e2e * (k + m) * L / e2e_t / 1e9
    if not torch.equal(h_par[0].cuda(), parity[0]) or not torch.equal(h_par[S_e2e - 1].cuda(), parity[S_e2e - 1]):
        raise RuntimeError("end-to-end parity differs from the device-resident parity")

    # The reference's own call shape: encode(&mut [T]) on one stripe of separately
    # allocated (pageable) shards, copies and kernel inside the timed call.
    single = {}
    rng_h = np.random.default_rng(5)
    for L1 in (65536, SHARD):
        shards = [rng_h.integers(0, 256, size=L1, dtype=np.uint8) for _ in range(k)]
        shards += [np.zeros(L1, np.uint8) for _ in range(m)]
        rs.encode(shards)
        reps = 40 if L1 == 65536 else 10
        t_start = time.perf_counter()
        for _ in range(reps):
            rs.encode(shards)
        t1s = (time.perf_counter() - t_start) / reps
        if not np.array_equal(shards[k][:64], device_parity_prefix(rs, shards, k, L1)):
            raise RuntimeError("single-stripe host encode differs from the device-resident encode")
        single["%d" % L1] = {"gbs": (k + m) * L1 / t1s / 1e9, "payload_mib_s": k * L1 / t1s / 2**20,
                             "ms_per_stripe": t1s * 1e3}

    hbm, hbm_kind = peaks()
    kern_avg = statistics.mean(kern_ms)
    achieved = bytes_per_step / (kern_avg * 1e-3) / 1e9
    traffic_per_stripe, traffic_src = profile_traffic()
    traffic = traffic_per_stripe * S if traffic_per_stripe else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform bytes, generated on device)",
            "config": {"workload": "RS(32,32) encode, 1 MiB shards, %d stripes per launch" % S,
                       "k": k, "m": m, "shard_bytes": L, "stripes_per_step": S,
                       "route": rs.encode_route(L), "l2": "inputs (%.0f GiB/step) larger than L2" % (S * k * L / 2**30),
                       "parallelism": "replicas over stripe partitions" if world > 1 else "1 GPU"},
            "frac_of_hbm": value / world / hbm,
            "plain": {"value": plain_gbs, "unit": "GB/s", "route": "matrix kernel, one stripe per launch",
                      "stripes": n_plain},
            "batched_over_plain": (value / world) / plain_gbs,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": "fft_kk_kernel<32> (one launch per step)",
                         "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % hbm_kind if hbm_kind == "measured"
                         else "fallback 6.65 TB/s", "traffic_source": traffic_src},
            "e2e": {"value": e2e_gbs, "unit": "GB/s", "h2d_bytes_per_step": S_e2e * k * L,
                    "d2h_bytes_per_step": S_e2e * m * L,
                    "path": "ReedSolomon.encode_batch_host (C ABI rs8_encode_batch) from pinned host memory",
                    "single_stripe_encode": dict(single, path="ReedSolomon.encode (C ABI rs8_encode), one stripe "
                                                 "of separately allocated pageable shards per call")},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if world == 1 and args.cpu_seconds > 0:  # 0 skips it (profiling runs)
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        if world == 1 and not args.no_extras:
            del data, parity
            torch.cuda.empty_cache()
            line["also"] = extras()
        print(json.dumps(line), flush=True)


def extras():
    """Other configurations measured in the same run, after the headline (each GB/s is
    algorithmic bytes over CUDA-event time; every reconstruct is checked bit-exact
    against the pre-erasure stripes): RS(32,32) reconstruct of 1 MiB shards with 1..m
    erasures per stripe, and the 10,000-stripe mixed batch (configuration 3) against one
    plain call per stripe."""
    from reed_solomon_b200 import workloads

    rec = workloads.stripes_sweep(shapes=((32, 32),), sizes=(SHARD,), n_stripes=256, reps=3)[0]
    mix = workloads.mixed_batch(n=10000, reps=3)
    return {
        "reconstruct_rs32x32_1MiB": {k2: rec[k2] for k2 in ("stripes", "reconstruct_gbs", "reconstruct_bit_exact",
                                                             "encode_fft_gbs", "encode_matrix_gbs")},
        "mixed_batch_10000": {k2: mix[k2] for k2 in ("stripes", "bytes", "batched_gbs", "batched_launches",
                                                      "plain_gbs", "batched_over_plain", "create_s",
                                                      "batched_matrix_only_gbs", "model_gbs", "exhaustive_gbs",
                                                      "regret_model", "regret_default") if k2 in mix},
    }


def run_workload(args):
    """The non-headline workloads: one JSON line with the workload's results."""
    import torch

    import __graft_entry__

    rsb = __graft_entry__.load_package()
    torch.cuda.set_device(0)
    from reed_solomon_b200 import workloads

    hbm, hbm_kind = peaks()
    launches0 = rsb.kernel_launch_count()
    with Clocks(0) as clk:
        if args.workload == "stripes":
            kw = {"n_stripes": args.stripes_count}
            if args.stripes_shapes:
                kw["shapes"] = tuple(tuple(int(x) for x in sh.split(",")) for sh in args.stripes_shapes.split("/"))
            if args.stripes_sizes:
                kw["sizes"] = tuple(int(x) for x in args.stripes_sizes.split(","))
            res = workloads.stripes_sweep(**kw)
            line = {"metric": "RS(k,m) encode/reconstruct GB/s, %d stripes per launch" % args.stripes_count,
                    "unit": "GB/s", "results": res}
        elif args.workload == "mixed":
            res = workloads.mixed_batch(n=args.mixed_stripes, packed=args.mixed_packed)
            line = {"metric": "mixed-shape batch GB/s, batched+tuned vs plain", "unit": "GB/s",
                    "value": res["batched_gbs"], "results": res}
        elif args.workload == "rs16":
            if args.rs16:
                res = workloads.rs16_shapes(shapes=[tuple(int(x) for x in sh.split(","))
                                                    for sh in args.rs16.split("/")])
            else:
                res = workloads.rs16_shapes()
            line = {"metric": "ReedSolomon16 encode/reconstruct GB/s", "unit": "GB/s", "results": res}
        elif args.workload == "tuner":
            save_t = os.path.splitext(args.save_model)[0] + "_timings.npz" if args.save_model else None
            res = workloads.tuner_regret(n_workloads=args.tuner_workloads, save_model=args.save_model,
                                         save_timings=save_t)
            line = {"metric": "cost-model route/tile regret vs exhaustive tuning (held out)", "unit": "fraction",
                    "value": res["regret_model"], "higher_is_better": False, "results": res}
        else:
            res = workloads.serve_poisson(count=args.requests)
            # The 50k req/s stream is far beyond one GPU; also measure latency at 60% of
            # the completion rate it achieved, where queues stay short.
            rate = 0.6 * res["completed_rate"]
            res["at_60pct_capacity"] = workloads.serve_poisson(count=args.requests, rate=rate, seed=6)
            line = {"metric": "request server p50/p99 latency and GB/s, Poisson 50k req/s", "unit": "GB/s",
                    "value": res["gbs"], "results": res}
    line.update({"workload": args.workload, "n_gpus": 1, "data": "synthetic (seeded uniform bytes, on device)",
                 "hbm_peak_gbs": hbm, "hbm_peak_source": hbm_kind,
                 "gpu_launches": rsb.kernel_launch_count() - launches0, "clocks": clk.summary()})
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload != "encode":
        if args.impl == "reference" or int(os.environ.get("WORLD_SIZE", 1)) > 1:
            print(json.dumps({"impl": args.impl, "workload": args.workload,
                              "unavailable": "workload runs on one GPU, our implementation only"}))
            return
        run_workload(args)
        return
    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
