"""Benchmark: homomorphic multiplication with relinearisation and rescale
(HMult, the key-switching workload) at N = 2^16 on one B200.

Workload (the key-switching configuration): 24 q primes (~30 bit) + 8
auxiliary primes (31 bit), hybrid key switching with dnum = 3, top level.
A step is one HMult+relin+rescale of each of `--batch` independent
ciphertext pairs (all resident in HBM, inputs larger than L2).  Residues are
synthetic: uniform in [0, q) from a seed (ciphertexts and the key alike; the
arithmetic does not depend on their distribution).

Reported (one JSON line on rank 0):
  value      HMult/s with inputs resident in HBM, CUDA events, max over ranks
  e2e        the same through the C ABI with host buffers: each step copies
             the batch in from pinned host memory, runs, copies results out
  roofline   the kernel with the largest device time in the step, timed by
             CUDA events on the context stream around its launches (a
             second pass of the same steps), algorithmic bytes per launch
  cpu_baseline  the CPU oracle's HMult on the host cores (bounded sample)
  bootstrap  full-slot bootstrapping throughput at N = 2^16 (bootstraps/s;
             decoded precision with real keys: tests/boot_precision_n16.py)
  ks_engines  the same step with the ModUp / ModDown column passes on each
             engine (--ks-engine picks the measured one; default auto: the
             library times both engines on the first launch of each shape
             and keeps the faster)
  bconv_engines  base conversion on CUDA cores vs tcgen05 tensor cores
  ntt        forward + inverse NTT round trip, 24 primes, HBM fraction
`--impl reference` times the CPU implementation of the path (the oracle;
the reference itself has no CPU path and cannot be built here) on the same
configuration.
"""
import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cheddar-fhe_b200"))

PARAM_FILE = "keyswitch_l24_a8.json"
METRIC = "HMult+relin+rescale/s (keyswitch/s) at N=2^16, L=24, alpha=8, dnum=3"
UNIT = "HMult/s"


from replicas import barrier, env_rank, finish, init_group, job_throughput, max_over_ranks, rank_seed  # noqa: E402


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        import statistics
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples),
                "window": "the timed steps plus 1 s of the same step right after them"}


def cpu_baseline_run(max_seconds=20.0, reps=None):
    """Times the CPU oracle's HMult on the same configuration."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle as po
    p = po.load_param_json(os.path.join(ROOT, "cheddar-fhe_b200", "params", PARAM_FILE))
    o = po.Oracle(p)
    lvl = o.max_level
    a = [o.uniform(1, lvl), o.uniform(2, lvl)]
    b = [o.uniform(3, lvl), o.uniform(4, lvl)]
    kb = np.stack([o.uniform(10 + i, o.max_level, num_aux=o.alpha) for i in range(o.beta_max)])
    ka = np.stack([o.uniform(20 + i, o.max_level, num_aux=o.alpha) for i in range(o.beta_max)])
    o.hmult(lvl, a, b, (kb, ka), rescale=True)  # warm
    n = 0
    t0 = time.perf_counter()
    while True:
        o.hmult(lvl, a, b, (kb, ka), rescale=True)
        n += 1
        el = time.perf_counter() - t0
        if (reps is not None and n >= reps) or (reps is None and el > max_seconds / 2) or el > max_seconds:
            break
    return n / el, n, el


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    times = []
    for _ in range(args.warmup):
        cpu_baseline_run(reps=1)
    total_n, total_t = 0, 0.0
    for _ in range(args.steps):
        v, n, el = cpu_baseline_run(reps=1)
        total_n += n
        total_t += el
        times.append(el)
    value = total_n / total_t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": {"workload": "HMult+relin+rescale, N=2^16, L=24 q primes, "
                                                    "alpha=8 aux primes, dnum=3, top level", "batch": 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{total_n} HMults of the CPU oracle (OpenMP over limbs)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU implementation of this path (its evaluator runs only on "
                "the GPU: compiled from its sources with rmm / libtommath stand-ins, it is timed on the "
                "same GPU in the main arm's reference_gpu); the CPU arm is the oracle port of its "
                "algorithm",
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-boot", action="store_true", help="skip the bootstrapping measurement")
    ap.add_argument("--boot-batch", type=int, default=8)
    ap.add_argument("--boot-profile", action="store_true",
                    help="profiling aid: set up the bootstrapping workload, run two BootBatch calls of "
                         "--boot-batch ciphertexts (the second is the one to read in a launch list) and exit")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own sm_100a build on the same workloads")
    ap.add_argument("--ks-engine", default="auto", choices=["cuda", "tensor", "tensor_wide", "auto"],
                    help="base conversion inside the ModUp / ModDown column passes of the measured path")
    ap.add_argument("--hmult-only", action="store_true",
                    help="profiling aid: measure only the HMult step (value, e2e, roofline) and print its line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch
    import cheddar_b200 as chd

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = init_group(world, "nccl")

    if args.boot_profile:
        stream = torch.cuda.Stream()
        boot_bench(chd, args, stream, None, profile=True)
        return
    params = json.load(open(os.path.join(chd.PARAM_DIR, PARAM_FILE)))
    ctx = chd.Context(json.dumps(params), device=local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.ks_engine = ks_engine_id(chd, args)
    lvl = ctx.max_level
    nq = ctx.num_q(lvl)
    n = ctx.n
    beta = -(-ctx.L // ctx.alpha)
    primes = torch.tensor(chd_primes(ctx), dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(rank_seed(1234, rank))

    def uniform(rows, gidx):
        q = primes[gidx][:, None]
        r = torch.randint(0, 2 ** 62, (rows, n), generator=gen, device="cuda", dtype=torch.int64)
        return (r % q).to(torch.int32)

    qg = torch.tensor(ctx.gidx(*ctx.level_np(lvl), 0), device="cuda", dtype=torch.int64)
    kg = torch.tensor(ctx.gidx(*ctx.level_np(ctx.max_level), ctx.alpha), device="cuda", dtype=torch.int64)
    kb = torch.stack([uniform(len(kg), kg) for _ in range(beta)]).contiguous()
    ka = torch.stack([uniform(len(kg), kg) for _ in range(beta)]).contiguous()
    key = chd.EvaluationKey(ctx, kb, ka, on_device=True)
    B = args.batch
    ins = [[uniform(nq, qg) for _ in range(4)] for _ in range(B)]
    a_cts = [ctx.import_ct(lvl, [x[0], x[1]], on_device=True) for x in ins]
    b_cts = [ctx.import_ct(lvl, [x[2], x[3]], on_device=True) for x in ins]
    outs = [chd.Ciphertext(ctx) for _ in range(B)]
    torch.cuda.synchronize()

    def step():
        ctx.HMultBatch(a_cts, b_cts, key, rescale=True, res_list=outs)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # ---- timed region (device events on the launching stream) ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(torch.cuda.current_device())
    if dist:
        barrier(dist)
    torch.cuda.synchronize()
    with sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        # the timed steps last a few ms, less than the 200 ms sampling
        # interval: the same step keeps running, untimed, for another second
        # so that the clock record covers this load
        t_end = time.time() + 1.0
        while time.time() < t_end:
            for _ in range(20):
                step()
            torch.cuda.synchronize()
    ms = max_over_ranks(dist, ev0.elapsed_time(ev1), "cuda")
    ms_step = ms / args.steps
    value = job_throughput(world, B, args.steps, ms)

    # ---- end to end through the C ABI with host buffers ----
    e2e = e2e_run(ctx, chd, key, lvl, nq, n, B, args, stream, dist)

    # ---- kernel launches of the measured step (two streams) ----
    ctx.stage_timing(True)
    for _ in range(args.steps):
        step()
    launches = sum(nl for _, nl in ctx.stage_times().values())
    ctx.stage_timing(False)
    # ---- per-stage device timing of the one-stream pipeline (kernels one
    # after another, so that each stage's events time its own launches):
    # dominant kernel and its roofline ----
    ctx.stream_split = False
    for _ in range(3):
        step()  # the one-stream launch shapes tuned outside the timed spans
    ctx.stage_timing(True)
    for _ in range(args.steps):
        step()
    stages = ctx.stage_times()
    ctx.stage_timing(False)
    ctx.stream_split = True
    roof = roofline_from_stages(ctx, lvl, B, stages, args.steps)

    ks_cmp = bconv_cmp = ntt_cmp = hoist_mixed = w64 = boot = split_cmp = None
    if not args.hmult_only:
        # ---- the same step with the key switch on one stream ----
        split_cmp = stream_split_cmp(ctx, step, stream, args.steps)
        # ---- the same step with each column-pass engine ----
        ks_cmp = ks_engines(ctx, chd, step, stream, args.steps, B)
        ks_cmp["plain_vs_tensor_batched"] = plain_vs_batched_hmult(ctx, chd, key, a_cts, b_cts, outs, stream,
                                                                   args.steps)

        # ---- base conversion as a dense contraction: CUDA cores vs tensor cores ----
        bconv_cmp = bconv_engines(ctx, chd, stream)

        # ---- NTT round trip (forward + inverse), 24 primes ----
        ntt_cmp = ntt_bench(chd, stream)

        # ---- hoisted rotations and a mixed-level batch ----
        hoist_mixed = hoist_mixed_bench(ctx, chd, key, uniform, stream)
        # ---- the 64-bit word path ----
        try:
            w64 = w64_bench(chd, stream)
        except Exception as e:  # reported, not fatal: the headline is the 32-bit path
            w64 = {"failed": str(e)[:300]}

        # ---- full-slot bootstrapping at N = 2^16 ----
        boot = None if args.no_boot else boot_bench(chd, args, stream, dist)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "HMult+relin+rescale, N=2^16, L=24 q primes (30-bit), alpha=8 aux primes "
                               "(31-bit), dnum=3, top level", "batch_per_gpu": B,
                   "l2": "inputs larger than L2 (batch x 24 MB + 48 MB key)",
                   "parallelism": f"replicas x{world}"},
        "e2e": e2e, "roofline": roof, "clocks": sampler.summary(), "ks_engine": args.ks_engine,
        "ks_engines": ks_cmp, "bconv_engines": bconv_cmp, "ntt": ntt_cmp,
        "bootstrap": boot, "hoisted_and_mixed": hoist_mixed, "w64": w64, "stream_split": split_cmp,
        "gpu_launches": launches,
    }
    # the autotuner's choice per column-pass launch shape (largest source
    # count K, jobs, largest target count M) -> engine / target split
    line["config"]["autotuned_column_passes"] = [
        f"K{t['K']} jobs{t['jobs']} M{t['M']}: "
        f"{({0: 'cuda_core', 1: 'tensor_core', 3: 'tensor_core_wide', 4: 'tensor_core_wide_128regs'}).get(t['engine'], t['engine'])}"
        f"/split{t['split']}"
        for t in chd.ks_tuned_shapes()]
    # the row pass's choice per shape (ciphertexts, rows, mode) -> variant
    line["config"]["autotuned_row_passes"] = [
        f"cts{t['cts']} rows{t['rows']} mode{t['mode']}: "
        f"{({0: 'in_place_loads', 1: 'prefetch', 2: 'in_place_loads_4ctas'}).get(t['variant'], t['variant'])}"
        for t in chd.ks_rows_tuned_shapes()]
    if rank == 0 and world == 1 and not args.no_reference_gpu and not args.hmult_only:
        ref = reference_gpu_run(args)
        try:
            ref["hmult_ours_over_reference"] = value / ref["hmult"]["hmult_per_s"]
        except (KeyError, TypeError, ZeroDivisionError):
            pass
        try:
            ref["ntt_ours_over_reference"] = (ref["ntt"]["us_per_roundtrip"] /
                                              ntt_cmp["batched"]["us_per_round_trip"])
        except (KeyError, TypeError, ZeroDivisionError):
            pass
        try:
            ref["boot_ours_over_reference"] = (ref["bootstrap"]["hoisted"]["ms_per_boot"] / boot["ms_per_boot"])
        except (KeyError, TypeError, ZeroDivisionError):
            pass
        try:
            ref["hmult64_ours_over_reference"] = ref["hmult64"]["ms_per_hmult"] / w64["ms_per_hmult"]
        except (KeyError, TypeError, ZeroDivisionError):
            pass
        line["reference_gpu"] = ref
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.hmult_only:
        try:
            v, cnt, el = cpu_baseline_run(max_seconds=20.0)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"{cnt} HMults of the CPU oracle in {el:.1f} s "
                                              "(OpenMP over limbs, all host threads)"}
        except Exception as e:  # pragma: no cover
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(line))
    del outs, a_cts, b_cts, key
    ctx.close()
    finish(dist)
    return 0


def chd_primes(ctx):
    import json as _j
    p = _j.load(open(os.path.join(ROOT, "cheddar-fhe_b200", "params", PARAM_FILE)))
    ter = list(reversed(p.get("terminal_primes", [])))
    return ter + p["main_primes"] + p["auxiliary_primes"]


def e2e_run(ctx, chd, key, lvl, nq, n, B, args, stream, dist):
    """End to end through the library's API with host buffers: every step
    copies its B input pairs from pinned host memory, runs HMultBatch and
    reads its B results back.  Steps are double-buffered over three streams
    (host-to-device copy of step i+1, HMult of step i on the context stream,
    device-to-host read of step i-1), ordered by CUDA events, so the PCIe
    transfers in both directions overlap the arithmetic; the timed region runs
    from the first copy to the last read."""
    import torch
    words = nq * n
    nout = ctx.num_q(lvl - 1)
    host_in = [[torch.randint(0, 1 << 29, (4, nq, n), dtype=torch.int32).pin_memory() for _ in range(B)]
               for _ in range(2)]
    host_out = [[torch.empty((2, nout, n), dtype=torch.int32).pin_memory() for _ in range(B)] for _ in range(2)]
    dev_in = [[torch.empty((4, nq, n), dtype=torch.int32, device="cuda") for _ in range(B)] for _ in range(2)]
    a_cts = [[ctx.wrap_ct(lvl, [dev_in[s][i][0], dev_in[s][i][1]]) for i in range(B)] for s in range(2)]
    b_cts = [[ctx.wrap_ct(lvl, [dev_in[s][i][2], dev_in[s][i][3]]) for i in range(B)] for s in range(2)]
    outs = [[chd.Ciphertext(ctx) for _ in range(B)] for _ in range(2)]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()  # noqa: E731
    in_ready, computed, read_back = [ev(), ev()], [ev(), ev()], [ev(), ev()]
    used = [False, False]

    def step(i):
        s = i & 1
        with torch.cuda.stream(h2d):
            if used[s]:
                h2d.wait_event(computed[s])  # step i-2 has consumed this input set
            for k in range(B):
                dev_in[s][k].copy_(host_in[s][k], non_blocking=True)
            in_ready[s].record(h2d)
        stream.wait_event(in_ready[s])
        if used[s]:
            stream.wait_event(read_back[s])  # step i-2's results are on the host
        ctx.HMultBatch(a_cts[s], b_cts[s], key, rescale=True, res_list=outs[s])
        computed[s].record(stream)
        d2h.wait_event(computed[s])
        for k in range(B):
            bx, ax, _ = ptrs(chd, outs[s][k])
            hb = host_out[s][k]
            nb = hb[0].numel() * 4
            cuda_copy_d2h(hb[0].data_ptr(), bx, nb, d2h)
            cuda_copy_d2h(hb[1].data_ptr(), ax, nb, d2h)
        read_back[s].record(d2h)
        used[s] = True

    for i in range(4):
        step(i)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        barrier(dist)
    steps = max(8, args.steps)  # enough steps that the pipeline's fill and drain are a small part
    ev0.record(h2d)
    for i in range(steps):
        step(i)
    h2d.wait_event(read_back[(steps - 1) & 1])
    h2d.wait_event(read_back[(steps - 2) & 1])
    ev1.record(h2d)
    torch.cuda.synchronize()
    ms = max_over_ranks(dist, ev0.elapsed_time(ev1), "cuda")
    world = dist.get_world_size() if dist else 1
    # the PCIe bound of this pipeline: one step's host-to-device bytes at the
    # bandwidth of the same copies alone (no kernels, no reads back)
    h2d_bytes = B * 4 * words * 4
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(h2d):
        c0.record(h2d)
        for r in range(3):
            for k in range(B):
                dev_in[r & 1][k].copy_(host_in[r & 1][k], non_blocking=True)
        c1.record(h2d)
    torch.cuda.synchronize()
    h2d_gbs = 3 * h2d_bytes / (c0.elapsed_time(c1) / 1e3) / 1e9
    value = job_throughput(world, B, steps, ms)
    bound = world * B / (h2d_bytes / (h2d_gbs * 1e9))  # every rank has its own link
    return {"value": value, "unit": UNIT,
            "h2d_bytes_per_step": h2d_bytes,
            "d2h_bytes_per_step": B * 2 * nout * n * 4,
            "pipeline": "double-buffered: H2D of step i+1, HMult of step i, D2H of step i-1 on three streams",
            "pcie_h2d_GB/s": h2d_gbs, "pcie_bound_hmult_per_s": bound, "frac_of_pcie_bound": value / bound}


_cudart = None


def cuda_copy_d2h(dst, src, nbytes, stream):
    import ctypes
    global _cudart
    if _cudart is None:
        import torch  # noqa: F401  (loads libcudart)
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                _cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        _cudart.cudaMemcpyAsync.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                            ctypes.c_void_p]
    rc = _cudart.cudaMemcpyAsync(ctypes.c_void_p(dst), ctypes.c_void_p(src), nbytes, 2,
                                 ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError(f"cudaMemcpyAsync failed: {rc}")


def ptrs(chd, ct):
    import ctypes
    bx, ax, rx = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    chd._check(chd.lib().chd_ct_device_ptrs(ct.ptr, ctypes.byref(bx), ctypes.byref(ax), ctypes.byref(rx)))
    return bx.value, ax.value, rx.value


def stage_limbs(ctx, lvl, batch):
    """Algorithmic limbs (N x u32 = 256 KiB each) one bench step moves per
    fused key-switch stage: every operand read once, every result written
    once; twiddles and tables excluded.  Returns {stage: (per-ciphertext
    limbs, per-launch limbs)}: the key is read once per key-switch row
    launch whatever the batch."""
    nq = ctx.num_q(lvl)
    tot = nq + ctx.alpha
    beta = -(-nq // ctx.alpha)          # digits at the top level (no terminal primes)
    dst = ctx.num_q(lvl - 1)            # ModDownAndRescale keeps the next level's primes
    drop = tot - dst
    return {
        "modup_inv_rows": (2 * nq + nq, 0),                  # a1, a2 in; a1*a2 rows out
        "modup_cols": (nq + beta * tot - nq, 0),             # digit sources in; other primes out
        "ks_rows": ((beta * tot - nq) + 4 * nq + 2 * tot,    # ModUp outputs, b1 a1 b2 a2, accumulators
                    2 * beta * tot),                         # key (bx, ax) per launch
        "moddown_cols": (2 * drop + 2 * dst, 0),             # dropped rows in; BConv+NTT out
        "fwd_rows_epilogue": (2 * dst + 2 * dst + 2 * dst, 0),  # BConv rows, kept accumulators in; out
    }


def roofline_from_stages(ctx, lvl, batch, stages, steps):
    """Roofline of the stage with the largest device time: algorithmic bytes
    per launch / average launch duration (CUDA events on the context stream,
    around each stage's launches inside the bench step)."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    limbs = stage_limbs(ctx, lvl, batch)
    limb_bytes = ctx.n * 4
    name = max(stages, key=lambda k: stages[k][0])
    ms_total, nl = stages[name]
    per_ct, per_launch = limbs[name]
    launches_per_step = nl / steps
    algo = (per_ct * batch / launches_per_step + per_launch) * limb_bytes
    ms = ms_total / nl
    achieved = algo / (ms / 1e3) / 1e9
    traffic, traffic_note = ncu_traffic(name, batch)
    return {"kernel": KERNEL_OF_STAGE[name], "bound": "hbm", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
            "traffic_source": traffic_note,
            "algorithmic_bytes_per_launch": algo, "ms_per_launch": ms,
            "stage_ms_per_step": {k: v[0] / steps for k, v in stages.items()},
            "stage_launches_per_step": {k: v[1] / steps for k, v in stages.items()}}


def ks_engine_id(chd, args):
    return {"cuda": chd.BCONV_CUDA_CORE, "tensor": chd.BCONV_TENSOR_CORE, "tensor_wide": chd.BCONV_TENSOR_CORE_WIDE,
            "auto": chd.BCONV_AUTO}[args.ks_engine]


def ks_engines(ctx, chd, step, stream, steps, B):
    """The HMult step with the ModUp / ModDown column passes on each engine
    (CUDA-core int64 BConv vs tcgen05 INT8 byte-limb MMAs); residues are
    identical (tests), only the time differs.  The one-stream pipeline, so
    that the stage events time each column pass alone."""
    import torch
    old = ctx.ks_engine
    ctx.stream_split = False
    out = {}
    for name, e in (("cuda_core", chd.BCONV_CUDA_CORE), ("tensor_core", chd.BCONV_TENSOR_CORE),
                    ("tensor_core_wide", chd.BCONV_TENSOR_CORE_WIDE), ("auto", chd.BCONV_AUTO)):
        ctx.ks_engine = e
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ctx.stage_timing(True)
        for _ in range(steps):
            step()
        st = ctx.stage_times()
        ctx.stage_timing(False)
        out[name] = {"hmult_per_s": B * steps / (ms / 1e3), "ms_per_step": ms / steps,
                     "modup_cols_ms": st["modup_cols"][0] / steps, "moddown_cols_ms": st["moddown_cols"][0] / steps}
    ctx.ks_engine = old
    ctx.stream_split = True
    out["speedup_tensor_vs_cuda_core"] = out["tensor_core"]["hmult_per_s"] / out["cuda_core"]["hmult_per_s"]
    out["speedup_tensor_wide_vs_cuda_core"] = (out["tensor_core_wide"]["hmult_per_s"] /
                                               out["cuda_core"]["hmult_per_s"])
    cols = {k: out[k]["modup_cols_ms"] + out[k]["moddown_cols_ms"] for k in ("cuda_core", "tensor_core",
                                                                           "tensor_core_wide")}
    out["column_pass_speedup"] = cols["cuda_core"] / cols["tensor_core"]
    out["column_pass_speedup_wide"] = cols["cuda_core"] / cols["tensor_core_wide"]
    return out


def stream_split_cmp(ctx, step, stream, steps):
    """The measured step with the fused key switch split over two streams
    (the default: halves of the batch on the context stream and on the
    context's second stream) and on the context stream alone; CUDA events on
    the context stream, which joins the second stream at the end of every
    key switch."""
    import torch
    res = {}
    for name, on in (("one_stream", False), ("two_streams", True)):
        ctx.stream_split = on
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        res[name + "_ms"] = e0.elapsed_time(e1) / steps
    ctx.stream_split = True
    res["speedup"] = res["one_stream_ms"] / res["two_streams_ms"]
    return res


def plain_vs_batched_hmult(ctx, chd, key, a_cts, b_cts, outs, stream, steps):
    """The two forms the design targets compare, same B pairs:
    plain = one HMult call per pair, CUDA-core column passes, eager launches;
    tensor-core batched = one HMultBatch over all B on the tensor-core
    engine, captured once as a CUDA graph and replayed."""
    import torch
    old = ctx.ks_engine
    B = len(a_cts)

    def timed(fn):
        for _ in range(3):
            fn()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ctx.ks_engine = chd.BCONV_CUDA_CORE

    def plain():
        for i in range(B):
            ctx.HMult(a_cts[i], b_cts[i], key, rescale=True, res=outs[i])

    ms_plain = timed(plain)
    ctx.ks_engine = chd.BCONV_TENSOR_CORE
    ctx.HMultBatch(a_cts, b_cts, key, rescale=True, res_list=outs)
    ctx.synchronize()
    ctx.graph_begin()
    ctx.HMultBatch(a_cts, b_cts, key, rescale=True, res_list=outs)
    graph = ctx.graph_end()
    ms_tc = timed(graph.launch)
    del graph
    ctx.ks_engine = old
    return {"plain_cuda_core_one_by_one": {"hmult_per_s": B / (ms_plain / 1e3), "ms_per_step": ms_plain},
            "tensor_core_batched_graph": {"hmult_per_s": B / (ms_tc / 1e3), "ms_per_step": ms_tc},
            "speedup": ms_plain / ms_tc}


NTT_PARAM_FILE = "ntt_bootparam30_p24.json"


def ntt_bench(chd, stream, counts=(32, 1), reps=10):
    """Negacyclic NTT round trip (forward, then inverse) at N = 2^16 over the
    24 primes main_primes[2..25] of the reference's bootparam_30.json
    (params/ntt_bootparam30_p24.json), `count` polynomials per launch pair:
    32 (32 x 24 limbs = 201 MB, larger than L2) for throughput, and 1 for
    the single-polynomial latency.  Uniform residues from a seed; the round
    trip must return the input unchanged.  Algorithmic bytes per
    polynomial: 2 transforms x (read + write) x 24 limbs x 256 KiB =
    25.17 MB."""
    import torch
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    params = json.load(open(os.path.join(chd.PARAM_DIR, NTT_PARAM_FILE)))
    ctx = chd.Context(json.dumps(params), device=torch.cuda.current_device())
    ctx.set_stream(stream.cuda_stream)
    lvl = ctx.max_level
    m, t = ctx.level_np(lvl)
    n = ctx.n
    allp = torch.tensor(params["main_primes"], dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(0)
    q = allp[None, :m, None]
    out = {"params": f"{NTT_PARAM_FILE}: main_primes[2..25] of the reference's bootparam_30.json"}
    for count in counts:
        x = (torch.randint(0, 2 ** 62, (count, m + t, n), generator=gen, device="cuda", dtype=torch.int64) % q)
        x = x.to(torch.int32).contiguous()
        ref = x.clone()
        torch.cuda.synchronize()

        def trip():
            ctx.ntt_raw(m, t, 0, x, mont=True, count=count)
            ctx.intt_raw(m, t, 0, x, mont=True, count=count)

        for _ in range(3):
            trip()
        ctx.synchronize()
        r = reps if count > 1 else 10 * reps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(r):
            trip()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / (r * count)  # per polynomial round trip
        exact = bool(torch.equal(x, ref))
        nbytes = 2 * 2 * (m + t) * n * 4
        key = "batched" if count > 1 else "one_polynomial"
        out[key] = {"workload": f"NTT + INTT round trip, N=2^16, {m + t} primes, {count} polys per launch pair",
                    "round_trips_per_s": 1e3 / ms, "us_per_round_trip": 1e3 * ms,
                    "GB/s": nbytes / (ms * 1e-3) / 1e9, "hbm_frac": nbytes / (ms * 1e-3) / 1e9 / hbm,
                    "algorithmic_bytes_per_round_trip": nbytes, "round_trip_exact": exact}
        del x, ref
    ctx.close()
    return out


def reference_gpu_run(args):
    """The reference's own evaluator (its sources compiled for sm_100a,
    oracle/_ref/libcheddar_ref.so) timed on this GPU on the same workloads:
    HMult+relin+rescale at the top level of the key-switching set (`batch`
    distinct pairs per step, one HMult per call: the reference has no
    batched entry point), the 24-prime NTT round trip, and full-slot
    bootstrapping of bootparam_40.json (hoisted and min-KS), and the 64-bit
    word path's HMult on bootparam_40_64bit.json.  Each workload
    runs in its own process (the reference keeps per-parameter-set state
    process-wide); CUDA events on the legacy stream the reference uses."""
    script = os.path.join(ROOT, "oracle", "ref_bench.py")
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcheddar_ref.so")):
        return {"unavailable": "oracle/_ref/libcheddar_ref.so not built"}
    jobs = [("hmult", ["hmult", PARAM_FILE, str(args.batch), str(max(args.steps, 10)), "3"]),
            ("ntt", ["ntt", "24", "32", "10", "3"]),
            ("ntt_one_polynomial", ["ntt", "24", "1", "100", "3"])]
    if not args.no_boot:
        jobs.append(("bootstrap", ["boot", BOOT_PARAM_FILE, "5", "2"]))
    jobs.append(("hmult64", ["hmult64", W64_PARAM_FILE, "20", "3"]))
    out = {"build": "the reference's src/core, src/extension, src/UserInterface.cu compiled for sm_100a "
                    "(oracle/Makefile target ref) with project-written rmm / libtommath stand-ins"}
    for name, argv in jobs:
        try:
            r = subprocess.run([sys.executable, script] + argv, capture_output=True, text=True, timeout=1200)
            lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out[name] = json.loads(lines[-1]) if r.returncode == 0 and lines else \
                {"failed": f"rc {r.returncode}: {r.stderr[-300:]}"}
        except Exception as e:  # pragma: no cover
            out[name] = {"failed": str(e)}
    return out


def bconv_engines(ctx, chd, stream, npoly=64, reps=10):
    """Base conversion of 64 polynomials at N = 2^16, ModUp 12 -> 4 (12 q
    primes extended by 4 auxiliary primes) and ModDown 4 -> 12, on the CUDA
    cores (int64 multiply-adds) and on the tcgen05 tensor cores (INT8 4-limb
    GEMM, int32 accumulation); outputs compared for equality.  Inputs are
    centred uniform residues, larger than L2 (64 x 16 limbs = 268 MB per
    direction).  Algorithmic bytes: every source limb read once, every
    target limb written once."""
    import torch
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    n = ctx.n
    main = list(range(12))
    aux = list(range(ctx.L, ctx.L + 4))
    gen = torch.Generator(device="cuda").manual_seed(99)
    res = {"workload": "BConv, 64 polys, N=2^16, ModUp 12->4 and ModDown 4->12", "engines_equal": True}
    for name, src, dst in (("modup_12_to_4", main, aux), ("moddown_4_to_12", aux, main)):
        K, M = len(src), len(dst)
        xt = torch.randint(-(1 << 29), 1 << 29, (npoly, K, n), generator=gen, device="cuda", dtype=torch.int32)
        outs = {}
        row = {}
        for eng_name, eng in (("cuda_core", chd.BCONV_CUDA_CORE), ("tensor_core", chd.BCONV_TENSOR_CORE)):
            out = torch.zeros((npoly, M, n), dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            for _ in range(3):
                ctx.bconv_batch(xt, src, dst, out, engine=eng, npoly=npoly)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                ctx.bconv_batch(xt, src, dst, out, engine=eng, npoly=npoly)
            e1.record(stream)
            ctx.synchronize()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            algo = npoly * (K + M) * n * 4
            entry = {"ms": ms, "GB/s": algo / (ms / 1e3) / 1e9, "hbm_frac": algo / (ms / 1e3) / 1e9 / hbm}
            if eng == chd.BCONV_TENSOR_CORE:
                ks = (4 * K + 31) // 32
                nb = max(16, (4 * M + 15) // 16 * 16)
                ops = 2 * npoly * n * ks * 32 * nb  # int8 multiply-adds issued, x2
                entry["int8_tops"] = ops / (ms / 1e3) / 1e12
                entry["int8_frac_of_nominal_4500"] = ops / (ms / 1e3) / 1e12 / 4500.0
            row[eng_name] = entry
            outs[eng_name] = out
        res["engines_equal"] = res["engines_equal"] and bool(torch.equal(outs["cuda_core"], outs["tensor_core"]))
        row["speedup_tensor_vs_cuda_core"] = row["cuda_core"]["ms"] / row["tensor_core"]["ms"]
        res[name] = row
    return res


def hoist_mixed_bench(ctx, chd, key, uniform, stream, reps=5):
    """(i) One ciphertext at the top level rotated by the 30 distinct offsets
    {+-2^k, k < 15} u {1..4} mod 2^15: all rotations of one ModUp in one
    launch (HoistedRotate, results in Q u P, then one batched ModDown of
    the 30 results) against 30 separate HRot calls.  (ii) 16 HMult+relin+rescale pairs at levels drawn
    uniformly from 5..22 (seed 0; 22 is this set's top level): one HMult
    call per pair, the batched call (one fused pipeline over every level:
    a launch per stage, the row pass taking up to 8 levels per launch), and
    the batched call captured once in a CUDA graph and replayed.  Keys are
    uniform random residues; CUDA events on the context stream."""
    import numpy as np
    import torch
    n, L, a = ctx.n, ctx.L, ctx.alpha
    beta = -(-L // a)
    lvl = ctx.max_level
    kg = torch.tensor(ctx.gidx(*ctx.level_np(lvl), a), device="cuda", dtype=torch.int64)
    offsets = sorted({(1 << k) % (n // 2) for k in range(15)} | {(-(1 << k)) % (n // 2) for k in range(15)} |
                     {1, 2, 3, 4})
    keys = []
    for _ in offsets:
        kb = torch.stack([uniform(len(kg), kg) for _ in range(beta)]).contiguous()
        ka = torch.stack([uniform(len(kg), kg) for _ in range(beta)]).contiguous()
        keys.append(chd.EvaluationKey(ctx, kb, ka, on_device=True))
    qg = torch.tensor(ctx.gidx(*ctx.level_np(lvl), 0), device="cuda", dtype=torch.int64)
    ct = ctx.import_ct(lvl, [uniform(len(qg), qg), uniform(len(qg), qg)], on_device=True)
    qp_outs = [chd.Ciphertext(ctx) for _ in offsets]
    outs = [chd.Ciphertext(ctx) for _ in offsets]

    def timed(fn):
        for _ in range(2):
            fn()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def hoisted():
        ctx.HoistedRotate(ct, keys, offsets, outs=qp_outs)
        ctx.ModDownBatch(qp_outs, res_list=outs)

    def separate():
        for k, r, o in zip(keys, offsets, outs):
            ctx.HRot(ct, k, r, res=o)

    ms_h = timed(hoisted)
    ms_s = timed(separate)
    # the two halves of the hoisted form on their own: the ModUp plus the
    # one rotation launch (results in Q u P), and the batched ModDown
    ms_rot = timed(lambda: ctx.HoistedRotate(ct, keys, offsets, outs=qp_outs))
    ms_md = timed(lambda: ctx.ModDownBatch(qp_outs, res_list=outs))
    R = len(offsets)
    # algorithmic limbs: the input (2 q), every rotation key once
    # (2 beta (q + alpha)) and every rotated result (2 q)
    nq = ctx.num_q(lvl)
    tot = nq + a
    limbs = 2 * nq + R * 2 * beta * (nq + a) + R * 2 * nq
    algo = limbs * n * 4
    # the rotation half: ModUp (read q, write beta (q + alpha)), P b (read
    # and write q), k_hoisted (read the beta digits, P b and every key,
    # write 2 (q + alpha) per rotation); the ModDown half: read 2 (q +
    # alpha), write 2 q per rotation
    rot_limbs = (nq + beta * tot) + 2 * nq + (beta * tot + nq + R * 2 * beta * tot + R * 2 * tot)
    md_limbs = R * 2 * tot + R * 2 * nq
    hbm = _peaks().get("hbm_gbs", 6650.0)
    res = {"hoisted_rotations": {
        "workload": f"{R} rotations of one ciphertext at level {lvl} (N=2^16, L=24, alpha=8)",
        "offsets": R, "hoisted_ms": ms_h, "separate_ms": ms_s,
        "hoisted_rotations_per_s": R / (ms_h / 1e3), "separate_rotations_per_s": R / (ms_s / 1e3),
        "speedup": ms_s / ms_h, "algorithmic_limbs": limbs, "algorithmic_bytes": algo,
        "hoisted_GB/s": algo / (ms_h / 1e3) / 1e9, "hoisted_hbm_frac": algo / (ms_h / 1e3) / 1e9 / hbm,
        "separate_hbm_frac": algo / (ms_s / 1e3) / 1e9 / hbm,
        "rotate_half": {"ms": ms_rot, "algorithmic_limbs": rot_limbs,
                        "hbm_frac": rot_limbs * n * 4 / (ms_rot / 1e3) / 1e9 / hbm},
        "moddown_half": {"ms": ms_md, "algorithmic_limbs": md_limbs,
                         "hbm_frac": md_limbs * n * 4 / (ms_md / 1e3) / 1e9 / hbm}}}
    del keys, qp_outs, outs
    # (ii) mixed-level batch
    levels = [int(x) for x in np.random.default_rng(0).integers(5, 23, 16)]

    def ct_at(level):
        g = torch.tensor(ctx.gidx(*ctx.level_np(level), 0), device="cuda", dtype=torch.int64)
        return ctx.import_ct(level, [uniform(len(g), g), uniform(len(g), g)], on_device=True)

    A = [ct_at(x) for x in levels]
    Bc = [ct_at(x) for x in levels]
    outs = [chd.Ciphertext(ctx) for _ in levels]

    def one_by_one():
        for x, y, o in zip(A, Bc, outs):
            ctx.HMult(x, y, key, rescale=True, res=o)

    def batched():
        ctx.HMultBatch(A, Bc, key, rescale=True, res_list=outs)

    ms_1 = timed(one_by_one)
    ms_b = timed(batched)
    ctx.synchronize()
    ctx.graph_begin()
    batched()
    graph = ctx.graph_end()
    ms_g = timed(graph.launch)
    del graph
    res["mixed_level_batch"] = {
        "workload": "16 HMult+relin+rescale pairs, levels U(5..22) seed 0, N=2^16, alpha=8",
        "levels": levels, "one_by_one_ms": ms_1, "batched_ms": ms_b, "graph_ms": ms_g,
        "hmult_per_s": {"one_by_one": 16 / (ms_1 / 1e3), "batched": 16 / (ms_b / 1e3),
                        "graph": 16 / (ms_g / 1e3)}}
    return res


BOOT_PARAM_FILE = "bootparam_40.json"
W64_PARAM_FILE = "bootparam_40_64bit.json"


def w64_bench(chd, stream, steps=20, warmup=3):
    """The 64-bit word path: HMult+relin+rescale of one pair at the top level
    of the reference's bootparam_40_64bit.json (26 main primes of 40-55 bits,
    7 auxiliary of 56 bits, dnum 4), uniform ciphertexts and key from the
    generator and seed the reference's timing uses, CUDA events on the stream
    the context runs on, the result buffer reused."""
    import numpy as np
    import torch
    p = json.load(open(os.path.join(chd.PARAM_DIR, W64_PARAM_FILE)))
    g = chd.Context64(json.dumps(p))
    g.set_stream(stream.cuda_stream)
    n = g.n
    primes = [int(x) for x in g.primes()]
    na, L = len(p["auxiliary_primes"]), len(p["main_primes"]) + len(p.get("terminal_primes", []))
    rng = np.random.default_rng(1)

    def uni(rows):
        return np.stack([rng.integers(0, primes[r], n, dtype=np.uint64) for r in rows])
    beta = -(-L // na)
    key = (np.stack([uni(range(L + na)) for _ in range(beta)]), np.stack([uni(range(L + na)) for _ in range(beta)]))
    a = (uni(range(L)), uni(range(L)))
    b = (uni(range(L)), uni(range(L)))
    lvl = g.max_level
    ga, gb = g.import_ct(lvl, a), g.import_ct(lvl, b)
    k = chd.EvaluationKey64(g, key[0], key[1])
    r = chd.Ciphertext64(g)
    for _ in range(warmup):
        g.HMult(ga, gb, k, True, res=r)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.HMult(ga, gb, k, True, res=r)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    g.set_stream(None)
    return {"workload": f"64-bit word path: HMult+relin+rescale at the top level of {W64_PARAM_FILE}",
            "ms_per_hmult": ms, "hmult_per_s": 1e3 / ms, "steps": steps,
            "kernels": "unfused: two-pass NTT, exact 128-bit base conversion, element-wise"}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def boot_trace_limbs(ctx, bc, params):
    """Algorithmic limbs (N-word polynomials) of one bootstrap: the sum over
    its op trace (the compiled Boot program, op for op as the library and
    the reference run it) of every operand read once and every result
    written once.  Per op at level l, with q = num_q(l), beta(l) digits and
    alpha auxiliary primes:
      key switch (RelinearizeRescale, HConj, HRotAdd): inputs, the key rows
        it reads (2 beta (q + alpha)), the result;
      linear transform: input 2q, one key per nonzero baby / giant step,
        every plaintext diagonal (q + alpha), result 2 q(l - 1);
      ModUpToMax: 2 q(-1) in, 2 q(max) out (+ the dense-to-sparse and
        sparse-to-dense key rows with encapsulation);
      element-wise, rescale, level-down, tensor: inputs and result.
    Returns (ciphertext-data limbs, key + plaintext limbs): a batch of B
    bootstraps reads the second part once in an ideal schedule."""
    prog = bc.json()
    lts = bc.transforms()
    a = ctx.alpha
    max_ter = len(params.get("terminal_primes", []))

    def q(l):
        return ctx.num_q(l)

    def key(l):
        m, t = ctx.level_np(l)
        beta = -(-(m + t + max_ter - t) // a)
        return 2 * beta * (q(l) + a)

    regs = {prog["input"]: (0, 2)}  # register -> (level, parts)
    data = const = 0
    for op in prog["ops"]:
        k, d, x, y, lvl = op["k"], op["d"], op["a"], op["b"], op["l"]
        if k in (0, 7):  # constant multiply / level-down (product, then rescale)
            lx, px = regs[x]
            level = lx if k == 7 else lvl
            data += px * q(lx if k == 7 else level)
            out = (level - 1, px) if k == 7 else (level, px)
            data += out[1] * q(out[0])
            regs[d] = out
        elif k == 1:  # tensor
            data += 2 * q(lvl) * 2 + 3 * q(lvl)
            regs[d] = (lvl, 3)
        elif k == 2:  # constant accumulation
            nparts = 2
            for src in op["s"]:
                ls, ps = regs[src]
                data += min(ps, 2) * q(lvl)
            if op["p"] >= 0:
                nparts = regs[op["p"]][1]
                data += nparts * q(lvl)
            data += nparts * q(lvl)
            regs[d] = (lvl, nparts)
        elif k in (3, 8, 12):  # add constant, copy, times i
            lx, px = regs[x]
            data += 2 * px * q(lx)
            regs[d] = (lx, px)
        elif k in (4, 10):  # add / sub
            lx, px = regs[x]
            py = regs[y][1]
            data += (px + py + max(px, py)) * q(lx)
            regs[d] = (lx, max(px, py))
        elif k == 5:  # RelinearizeRescale
            lx, px = regs[x]
            data += px * q(lx) + 2 * q(lx - 1)
            const += key(lx)
            regs[d] = (lx - 1, 2)
        elif k == 6:  # rescale
            lx, px = regs[x]
            data += px * (q(lx) + q(lx - 1))
            regs[d] = (lx - 1, px)
        elif k in (9, 16):  # metadata
            pass
        elif k == 11:  # HConj
            lx, _ = regs[x]
            data += 4 * q(lx)
            const += key(lx)
            regs[d] = (lx, 2)
        elif k == 13:  # ModUpToMax
            top = ctx.max_level
            lx, _ = regs[x]
            data += 2 * q(lx) + 2 * q(top)
            if params.get("dense_hamming_weight") != params.get("sparse_hamming_weight"):
                const += 2 * (2 * q(-1)) + 2 * (q(top) + a)
            regs[d] = (top, 2)
        elif k == 14:  # HRotAdd
            lx, _ = regs[x]
            data += 6 * q(lx)
            const += key(lx)
            regs[d] = (lx, 2)
        elif k == 15:  # linear transform
            plan = lts[op["r"]]
            l = plan["level"]
            bs = {b for (_, b, _) in plan["pts"]}
            gs = {g for (g, _, _) in plan["pts"]}
            data += 2 * q(l) + 2 * q(l - 1)
            const += (len([b for b in bs if b]) + len([g for g in gs if g])) * key(l)
            const += len(plan["pts"]) * (q(l) + a)
            regs[d] = (l - 1, 2)
        else:
            raise ValueError(f"unknown op kind {k}")
    return data, const


def boot_bench(chd, args, stream, dist, profile=False):
    """Full-slot bootstrapping (N = 2^16, 2^15 slots) on the reference's own
    bootparam_40.json (4 terminal + 43 main primes, max level 28, alpha = 12,
    sparse-secret encapsulation, 4 CoeffToSlot and 3 SlotToCoeff levels,
    EvalMod with the reference's cosine polynomial and 3 double angles).  A step bootstraps a batch of level-0 ciphertexts in one
    BootBatch call (key switches and linear transforms batched across the
    ciphertexts), captured once as a CUDA graph and replayed; the eager
    batched call and one Boot per ciphertext are timed too.  CUDA events on
    the context stream, inputs resident.
    The evaluation keys are uniform random residues (the work is that of
    real keys; decoded precision with the reference's own keys is measured
    by tests/test_gpu_refpin.py, whose bootstraps equal the reference's
    residue for residue)."""
    import torch
    params = json.load(open(os.path.join(chd.PARAM_DIR, BOOT_PARAM_FILE)))
    ctx = chd.Context(json.dumps(params), device=torch.cuda.current_device())
    ctx.set_stream(stream.cuda_stream)
    ctx.ks_engine = ks_engine_id(chd, args)
    t0 = time.time()
    bc = chd.BootContext(ctx)
    plan_s = time.time() - t0
    rots = sorted(set(bc.rotations()) | set(bc.rotations(min_ks=True)))
    n, L, a = ctx.n, ctx.L, ctx.alpha
    beta = -(-L // a)
    allp = torch.tensor(list(reversed(params.get("terminal_primes", []))) + params["main_primes"] +
                        params["auxiliary_primes"], dtype=torch.int64, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(4321)

    def uniform(rows_gidx):
        q = allp[torch.tensor(rows_gidx, device="cuda", dtype=torch.int64)][:, None]
        r = torch.randint(0, 2 ** 62, (len(rows_gidx), n), generator=gen, device="cuda", dtype=torch.int64)
        return (r % q).to(torch.int32)

    kg = list(ctx.gidx(*ctx.level_np(ctx.max_level), a))
    keys = chd.EvkMap(ctx)
    held = []

    def ukey():
        kb = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        ka = torch.stack([uniform(kg) for _ in range(beta)]).contiguous()
        k = chd.EvaluationKey(ctx, kb, ka, on_device=True)
        held.append(k)
        return k

    keys.set_mult(ukey())
    keys.set_conjugation(ukey())
    for r in rots:
        keys.set_rotation(r, ukey())
    if params["dense_hamming_weight"] != params["sparse_hamming_weight"]:
        # sparse-secret encapsulation: the dense-to-sparse key over the level
        # -1 primes and as many auxiliary primes, the sparse-to-dense key as
        # one digit over the whole key basis
        m1, t1 = ctx.level_np(-1)
        g_dts = list(ctx.gidx(m1, t1, m1 + t1))
        held.append(chd.EvaluationKey(ctx, uniform(g_dts)[None].contiguous(), uniform(g_dts)[None].contiguous(),
                                      on_device=True, basis=(m1, t1, m1 + t1)))
        keys.set_dense_to_sparse(held[-1])
        mm, tt = ctx.level_np(ctx.max_level)
        held.append(chd.EvaluationKey(ctx, uniform(kg)[None].contiguous(), uniform(kg)[None].contiguous(),
                                      on_device=True, basis=(mm, tt, a)))
        keys.set_sparse_to_dense(held[-1])
    g0 = list(ctx.gidx(*ctx.level_np(0), 0))
    B = args.boot_batch
    ins = [ctx.import_ct(0, [uniform(g0), uniform(g0)], on_device=True, scale=ctx.scale(0)) for _ in range(B)]
    outs = [chd.Ciphertext(ctx) for _ in range(B)]
    torch.cuda.synchronize()

    def step_single():
        for i in range(B):
            bc.Boot(ins[i], keys, res=outs[i])

    def step():
        # one batched call: every key switch / linear transform over all B
        bc.BootBatch(ins, keys, res_list=outs)

    if profile:
        # the first call tunes the column passes; the second, inside the
        # NVTX range "boot_batch", is the one a profiler should capture
        # (ncu --nvtx --nvtx-include "boot_batch/")
        step()
        ctx.synchronize()
        torch.cuda.nvtx.range_push("boot_batch")
        step()
        ctx.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"boot_profile": "2 BootBatch calls", "batch": B}))
        return None

    for _ in range(2):
        step()
        step_single()
    ctx.synchronize()
    steps = max(1, min(args.steps, 5))
    # one ciphertext per call, for comparison
    es0, es1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es0.record(stream)
    for _ in range(steps):
        step_single()
    es1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_single = es0.elapsed_time(es1)
    # the plain form: one ciphertext per call on the CUDA-core engine
    main_engine = ctx.ks_engine
    ctx.ks_engine = chd.BCONV_CUDA_CORE
    step_single()
    ctx.synchronize()
    es0.record(stream)
    for _ in range(steps):
        step_single()
    es1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_plain = es0.elapsed_time(es1)
    # one ciphertext per call with the autotuned engine
    ctx.ks_engine = chd.BCONV_AUTO
    step_single()
    ctx.synchronize()
    es0.record(stream)
    for _ in range(steps):
        step_single()
    es1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_single_auto = es0.elapsed_time(es1)
    ctx.ks_engine = main_engine
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), "cuda")
    world = dist.get_world_size() if dist else 1
    # graph-captured batch (the configuration's form): the B bootstraps of a
    # step captured once as a CUDA graph and replayed
    ctx.graph_begin()
    step()
    graph = ctx.graph_end()
    graph.launch()
    ctx.synchronize()
    eg0, eg1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eg0.record(stream)
    for _ in range(steps):
        graph.launch()
    eg1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_graph = max_over_ranks(dist, eg0.elapsed_time(eg1), "cuda")
    del graph
    # the same graph-captured batch with every key switch and ModDown on the
    # context stream alone
    ctx.stream_split = False
    step()
    ctx.synchronize()
    ctx.graph_begin()
    step()
    graph = ctx.graph_end()
    graph.launch()
    ctx.synchronize()
    eg0.record(stream)
    for _ in range(steps):
        graph.launch()
    eg1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_graph_one = max_over_ranks(dist, eg0.elapsed_time(eg1), "cuda")
    del graph
    ctx.stream_split = True
    # the min-KS form (two rotation keys per transform, Boot(..., min_ks=true))
    bc.BootBatch(ins, keys, res_list=outs, min_ks=True)
    ctx.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(steps):
        bc.BootBatch(ins, keys, res_list=outs, min_ks=True)
    e3.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_mk = e2.elapsed_time(e3)
    # the same bootstraps with each column-pass engine
    engines = {}
    main_engine = ctx.ks_engine
    for name, e in (("cuda_core", chd.BCONV_CUDA_CORE), ("tensor_core", chd.BCONV_TENSOR_CORE),
                    ("tensor_core_wide", chd.BCONV_TENSOR_CORE_WIDE), ("auto", chd.BCONV_AUTO)):
        ctx.ks_engine = e
        step()
        ctx.synchronize()
        e2.record(stream)
        for _ in range(steps):
            step()
        e3.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        t = e2.elapsed_time(e3)
        engines[name] = {"ms_per_boot": t / (B * steps), "bootstraps_per_s": B * steps / (t / 1e3)}
    ctx.ks_engine = main_engine
    engines["speedup_tensor_vs_cuda_core"] = (engines["tensor_core"]["bootstraps_per_s"] /
                                              engines["cuda_core"]["bootstraps_per_s"])
    engines["speedup_tensor_wide_vs_cuda_core"] = (engines["tensor_core_wide"]["bootstraps_per_s"] /
                                                   engines["cuda_core"]["bootstraps_per_s"])
    try:
        data_l, const_l = boot_trace_limbs(ctx, bc, params)
        hbm = _peaks().get("hbm_gbs", 6650.0)
        batch_bytes = (B * data_l + const_l) * n * 4
        one_bytes = (data_l + const_l) * n * 4
        roof = {"bound": "hbm", "unit": "GB/s", "peak": hbm,
                "achieved": batch_bytes / (ms_graph / steps / 1e3) / 1e9,
                "frac": batch_bytes / (ms_graph / steps / 1e3) / 1e9 / hbm,
                "algorithmic_bytes_per_batch": batch_bytes, "algorithmic_bytes_one_boot": one_bytes,
                "ciphertext_limbs_per_boot": data_l, "key_and_plaintext_limbs": const_l,
                "one_by_one_frac": one_bytes / (ms_single / (B * steps) / 1e3) / 1e9 / hbm,
                "what": "algorithmic bytes of the op trace (each operand read once, each result written once; "
                        "keys and plaintext diagonals once per batch) / graph-replayed batch time; peak = "
                        "measured HBM copy"}
    except Exception as e:  # pragma: no cover
        roof = {"error": f"trace count failed: {e}"}
    res = {"metric": "bootstraps/s (full slots, N=2^16, batched call, graph-captured)",
           "roofline": roof,
           "value": job_throughput(world, B, steps, ms_graph),
           "eager": {"bootstraps_per_s": world * B * steps / (ms / 1e3), "ms_per_boot": ms / (B * steps)},
           "one_by_one_eager": {"bootstraps_per_s": world * B * steps / (ms_single / 1e3),
                                "ms_per_boot": ms_single / (B * steps),
                                "ms_per_boot_auto_engine": ms_single_auto / (B * steps)},
           "plain_vs_tensor_batched": {
               "plain_cuda_core_one_by_one_ms_per_boot": ms_plain / (B * steps),
               "tensor_core_batched_graph_ms_per_boot": ms_graph / (B * steps),
               "speedup": ms_plain / ms_graph},
           "stream_split": {"one_stream_ms_per_boot": ms_graph_one / (B * steps),
                            "two_streams_ms_per_boot": ms_graph / (B * steps), "speedup": ms_graph_one / ms_graph},
           "min_ks": {"ms_per_boot": ms_mk / (B * steps), "bootstraps_per_s": B * steps / (ms_mk / 1e3),
                      "rotation_keys": len(bc.rotations(min_ks=True))},
           "unit": "bootstraps/s", "ms_per_boot": ms_graph / (B * steps), "batch_per_gpu": B, "steps": steps,
           "ks_engine": args.ks_engine, "ks_engines": engines,
           "warmup": 2, "params": f"{BOOT_PARAM_FILE}: the reference's own 40-bit bootstrapping parameter file "
                                  "(4 terminal + 43 main primes, max level 28, alpha=12, sparse-secret "
                                  "encapsulation), 4 CtS + 3 StC levels, EvalMod deg-30 Chebyshev cosine + 3 "
                                  "double angles",
           "rotation_keys": len(bc.rotations()), "plan_seconds": plan_s,
           "keys": "uniform random residues (same work as real keys)",
           "levels": {"cts_start": bc.cts_start, "eval_mod_start": bc.eval_mod_start,
                      "stc_start": bc.stc_start, "end": bc.end_level}}
    del ins, outs, keys, held
    ctx.close()
    return res


KERNEL_OF_STAGE = {
    "modup_inv_rows": "k_inv_rows16", "modup_cols": "k_modswitch_cols (ModUp)", "ks_rows": "k_ks_rows",
    "moddown_cols": "k_modswitch_cols (ModDown)", "fwd_rows_epilogue": "k_fwd_rows16",
}


# sources a stage's kernel is compiled from (cheddar-fhe_b200/csrc): a
# committed DRAM-traffic capture counts only while their fingerprint matches
KERNEL_SOURCES = {"ks_rows": ["keyswitch.cu", "arith.cuh", "ntt_common.cuh"]}


def kernel_fingerprint(stage):
    """First 12 hex digits of the SHA-256 over the stage kernel's source
    files, or None for a stage without a source list."""
    files = KERNEL_SOURCES.get(stage)
    if not files:
        return None
    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(ROOT, "cheddar-fhe_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:12]


def ncu_traffic(stage, batch):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    the stage's kernel at this batch, from the committed ncu summary
    profiles/traffic_hmult_l24.md (a line `traffic <stage> <batch> <bytes>
    <source fingerprint>`), and a note.  The bytes are None when no capture
    was made or when the kernel's sources changed after it (the fingerprint
    differs)."""
    try:
        for ln in open(os.path.join(ROOT, "profiles", "traffic_hmult_l24.md")):
            f = ln.strip().strip("`").split()
            if len(f) == 5 and f[0] == "traffic" and f[1] == stage and int(f[2]) == batch:
                if f[4] != kernel_fingerprint(stage):
                    return None, "the committed ncu capture predates the current kernel source"
                return float(f[3]), "ncu capture of this kernel source (fingerprint " + f[4] + ")"
    except (OSError, ValueError):
        pass
    return None, "no ncu capture of this kernel at this batch"


if __name__ == "__main__":
    sys.exit(main())
