"""Benchmark: batched complex matrix exponential over a frequency sweep.

Workload (one "step"): exp(A_k) for a sweep of 256 complex matrices
A_k = -(G_k + i w_k C_k), orders n_k uniform in [64, 1024], G_k nonsymmetric
N(0,1)/sqrt(n), C_k = Q^T D Q SPD with D log-uniform in [1e-3, 1], w_k
log-spaced 1e2..1e6 -- seeded synthetic data with the shapes and value
distributions of the batching configuration. Metric: expm/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): the job is one sweep of 256 x N
matrices, partitioned over the N ranks by LPT on the estimated cost
n^3 (log2 w + 8) (csharp_linearalgebra_b200.sweep); each rank builds and
runs its own part (weak scaling: 256 matrices' worth per GPU, no collective
on the data path) and the time is the max over ranks. --shard seeds gives
every rank its own 256-matrix sweep instead.

Two forms run on the same sweep. The split-precision form (`value`, `e2e`,
`roofline`) computes the Pade-evaluation and squaring products from 8-bit
residues modulo `--moduli` coprime moduli on the tcgen05 tensor cores; its
error against the plain form is reported per matrix next to the matrix's
own FP64 sensitivity floor (`split_accuracy`). The plain FP64 form
(`plain_fp64`), every product on the FP64 DMMA path, is bit-identical to the
reference. `value` has the inputs resident in HBM (device entry point); `e2e`
goes through the host-buffer entry point with pinned buffers, so every step
copies each matrix in and each exponential out. Rooflines: the split form's
8-bit product kernel against cuBLASLt int8 measured in the same process, the
plain form's DMMA GEMM against cuBLAS DGEMM (CUDA events on the library's
stream). `--impl reference` times the CPU restatement of the reference's
algorithm (the oracle) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched complex expm/s: split-prec vs plain FP64 GPU at ≤1e-12 rel err; vs CPU"
# DRAM bytes of the GEMM launches per algorithmic byte, from one ncu capture of every GEMM launch of
# the 16-matrix sweep (same generator, --count 16): 109.1 MB measured / 153.4 MB.
GEMM_TRAFFIC_RATIO = 109.1 / 153.35
# The same for the modular GEMM of the split form: every modular_gemm launch of the 16-matrix sweep
# (110 launches) read and wrote 105.59 GB of DRAM against 101.09 GB of algorithmic bytes.
SPLIT_TRAFFIC_RATIO = 105.585 / 101.086
WORKLOAD = ("frequency sweep of 256 complex128 matrices A_k = -(G + i w_k C), n_k ~ U{64..1024}, "
            "G ~ N(0,1)/sqrt(n), C = Q^T D Q (D log-uniform [1e-3,1]), w_k log-spaced 1e2..1e6; Expm of each")


def sweep_spec(count: int, seed: int):
    """Orders and frequencies of the seeded sweep: n_k ~ U{64..1024}, w_k
    log-spaced 1e2..1e6."""
    orders = np.random.default_rng(seed).integers(64, 1025, size=count)
    return [int(n) for n in orders], np.logspace(2.0, 6.0, count)


def sweep_matrix(k: int, n: int, w: float, seed: int):
    """Matrix k of the sweep, A = -(G + i w C), from its own seeded stream, so
    that any rank can build any subset of the sweep on its own."""
    rng = np.random.default_rng([seed, k])
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def make_sweep(count: int, seed: int, indices=None):
    """The seeded synthetic sweep (or the listed matrices of it): orders and
    complex128 Fortran arrays."""
    orders, omegas = sweep_spec(count, seed)
    idx = range(count) if indices is None else indices
    return [orders[k] for k in idx], [sweep_matrix(k, orders[k], omegas[k], seed) for k in idx]


def cpu_sample(count, size):
    """Indices of the bounded CPU sample: every ceil(count/size)-th matrix of
    the sweep, starting half a stride in, so that the sample spans the whole
    omega range (1e2..1e6, hence every squaring count) and the order range."""
    stride = max(1, -(-count // size))
    return list(range(stride // 2, count, stride))[:size]


def sample_chunks(sample, chunks):
    """The sample in `chunks` interleaved parts, each again spanning omega."""
    return [sample[c::chunks] for c in range(chunks) if sample[c::chunks]]


def expm_cost(n, s):
    """The cost model of one Expm: n^3 (s + 8), about the product count of
    degree 13 (six products, the Pade solve, s squarings) times n^3."""
    return float(n) ** 3 * (s + 8)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks_of(dist, value, device):
    """The largest of every rank's `value` (a step time): the slowest rank
    bounds a weak-scaling step. `dist` is torch.distributed or None (one rank);
    the tensor lives on `device` (CUDA for NCCL, CPU for gloo)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_arm(args, world, rank):
    """The reference's algorithm on the host cores (the oracle restatement),
    on the same stratified sample as the GPU arm's cpu_baseline. The sample's
    matrices are split into interleaved chunks, each spanning omega; step j
    runs chunk j mod chunks, so that a step stays bounded."""
    if rank != 0:
        return
    from oracle import oracle
    oracle.lib()
    threads = oracle.threads()
    orders, _ = sweep_spec(args.count, args.seed)
    sample = cpu_sample(len(orders), args.cpu_sample)
    mats = dict(zip(sample, make_sweep(args.count, args.seed, sample)[1]))
    chunks = sample_chunks(sample, args.ref_chunks)
    infos = {}

    def step(j):
        for i in chunks[j % len(chunks)]:
            _, info = oracle.expm(mats[i])
            infos[i] = info

    for w in range(args.warmup):
        step(w)
    done = 0
    t0 = time.perf_counter()
    for j in range(args.steps):
        step(j)
        done += len(chunks[j % len(chunks)])
    elapsed = time.perf_counter() - t0
    value = done / elapsed
    covered = sorted(set(i for j in range(args.steps) for i in chunks[j % len(chunks)]))
    squarings = [infos[i]["squarings"] for i in covered]
    desc = (f"stratified: every {sample[1] - sample[0] if len(sample) > 1 else 1}-th matrix of the sweep "
            f"({len(sample)} matrices, omega {min(OMEGAS(args.count)[i] for i in sample):.3g}.."
            f"{max(OMEGAS(args.count)[i] for i in sample):.3g}), in {len(chunks)} interleaved chunks; timed steps "
            f"covered {len(covered)} of them, orders {[orders[i] for i in covered]}, squarings {squarings}")
    line = {"metric": METRIC, "value": value, "unit": "expm/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex128)", "data": "synthetic, seeded",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "count": args.count, "seed": args.seed, "sample": desc,
                       "sample_cost_n3_s8": sum(expm_cost(orders[i], infos[i]["squarings"]) for i in covered),
                       "sweep_sum_n3": sum(float(n) ** 3 for n in orders)},
            "cpu_baseline": {"value": value, "unit": "expm/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "expm/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def OMEGAS(count):
    """The sweep's frequencies, as make_sweep draws them."""
    return np.logspace(2.0, 6.0, count)


def measured_fp64_peak(torch):
    """cuBLAS DGEMM TFLOP/s (burst) on this GPU, the FP64 denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_int8_peak(torch):
    """cuBLASLt 8-bit GEMM TOPS (burst, torch._int_mm 8192^3) on this GPU: the
    denominator of the split-precision kernel's roofline."""
    n = 8192
    try:
        a = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda")
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        del a, b
        torch.cuda.empty_cache()
        return best, "torch._int_mm (cuBLASLt int8) 8192^3 measured in this process"
    except Exception as exc:  # report the nominal figure, saying so
        return 4500.0, f"nominal dense INT8 4.5 POPS (measurement failed: {type(exc).__name__})"


def rel1_device(x, y):
    """||x - y||_1 / ||y||_1 for matrices stored transposed (row j = column j)."""
    return float((x - y).abs().sum(dim=1).max() / y.abs().sum(dim=1).max())


def ours(args, world, rank, local, dist):
    import torch
    torch.cuda.set_device(local)
    from csharp_linearalgebra_b200 import Workspace

    peak64 = None if args.no_peak else measured_fp64_peak(torch)
    peak8, peak8_src = (None, None) if args.no_peak else measured_int8_peak(torch)
    if args.shard == "lpt" and world > 1:
        from csharp_linearalgebra_b200.sweep import expm_cost_estimate, lpt_partition
        g_orders, g_omegas = sweep_spec(args.count * world, args.seed)
        parts, loads = lpt_partition([expm_cost_estimate(n, w) for n, w in zip(g_orders, g_omegas)], world)
        orders, mats = make_sweep(args.count * world, args.seed, parts[rank])
        shard_note = (f"one sweep of {args.count * world} matrices partitioned over {world} ranks by LPT on "
                      f"n^3 (log2 w + 8); rank loads within {100 * (max(loads) / min(loads) - 1):.2f}%")
    else:
        orders, mats = make_sweep(args.count, args.seed + 1000 * rank)
        shard_note = f"{world} rank(s), each its own {args.count}-matrix sweep"
    count = len(mats)
    # device-resident inputs and one set of outputs per form
    dev_in = [torch.from_numpy(m.T.copy()).to("cuda") for m in mats]  # row-major of A^T == column-major A
    a_ptrs = [t.data_ptr() for t in dev_in]
    in_bytes = sum(n * n * 16 for n in orders)
    # pinned host buffers for the end-to-end path
    host_in = [torch.from_numpy(m.T.copy()).pin_memory() for m in mats]
    host_out = [torch.empty_like(t).pin_memory() for t in host_in]
    hi_ptrs = [t.data_ptr() for t in host_in]
    ho_ptrs = [t.data_ptr() for t in host_out]

    ws = Workspace(local)
    ws.set_workers(args.groups)
    ws.set_autotune(bool(args.autotune))
    stream = torch.cuda.ExternalStream(ws.stream)
    if args.configs_only:
        # Only the other configurations' measurements (a profiling or a quick run).
        del host_in, host_out
        configs = other_configurations(args, ws, torch, peak64, peak8, (orders, mats, dev_in))
        if rank == 0:
            print(json.dumps({"configurations": configs}), flush=True)
        ws.dispose()
        return

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(ms):
        return max_over_ranks_of(dist, ms, "cuda")

    def run_form(moduli, inputs):
        """Warm-up, K timed steps (inputs in HBM), one single-group sweep timed
        launch by launch, and K end-to-end steps, all in one form."""
        ws.set_split_moduli(moduli)
        outs = [torch.empty_like(t) for t in inputs]
        ip = [t.data_ptr() for t in inputs]
        op = [t.data_ptr() for t in outs]

        def step():
            return ws.expm_batched_device(count, orders, ip, orders, op, orders)

        for _ in range(args.warmup):
            diags = step()
        torch.cuda.synchronize()
        ws.reset_stats()
        with ClockSampler(local) as clocks:
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                diags = step()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
        st_step = ws.stats()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        # The dominant kernels timed launch by launch with CUDA events on the
        # library's stream: one more sweep with a single group, so that no
        # other stream shares the GPU with a timed launch.
        ws.set_workers(1)
        ws.reset_stats()
        ws.set_timing(True)
        step()
        ws.set_timing(False)
        st = ws.stats()
        ws.set_workers(args.groups)
        return {"ms": ms, "st_step": st_step, "st": st, "clocks": clocks.summary(), "diags": diags,
                "e2e_ms": None, "outs": outs}

    def run_e2e(moduli):
        """K end-to-end steps through the host-buffer entry point."""
        ws.set_split_moduli(moduli)
        ws.expm_batched_host(count, orders, hi_ptrs, orders, ho_ptrs, orders)  # warm-up
        barrier()
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            ws.expm_batched_host(count, orders, hi_ptrs, orders, ho_ptrs, orders)
        e3.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e2.elapsed_time(e3) / args.steps)

    # Both forms' device-resident runs first (split, then plain), then both
    # end-to-end runs, so that no host-buffer pass reshapes the memory pool
    # between a form's warm-up and its timed steps.
    split = run_form(args.moduli, dev_in)
    plain = run_form(0, dev_in)
    if not args.no_e2e:
        split["e2e_ms"] = run_e2e(args.moduli)
        plain["e2e_ms"] = run_e2e(0)
    assert [(d.degree, d.squarings) for d in plain["diags"]] == [(d.degree, d.squarings) for d in split["diags"]]

    # Accuracy of the split form against the plain FP64 form (bit-identical to
    # the reference's result), next to each matrix's FP64 floor: how far the
    # plain result moves when the input moves by about one ulp.
    gen = torch.Generator(device="cuda").manual_seed(12345)
    pert = [t * (1.0 + 2.0 ** -52 * torch.randn(t.shape, dtype=torch.float64, device="cuda", generator=gen))
            for t in dev_in]
    ws.set_split_moduli(0)
    pert_out = [torch.empty_like(t) for t in pert]
    ws.expm_batched_device(count, orders, [t.data_ptr() for t in pert], orders, [t.data_ptr() for t in pert_out],
                           orders)
    torch.cuda.synchronize()
    errs = [rel1_device(s, p) for s, p in zip(split["outs"], plain["outs"])]
    floors = [rel1_device(q, p) for q, p in zip(pert_out, plain["outs"])]
    ratios = [e / f if f > 0 else (0.0 if e == 0 else float("inf")) for e, f in zip(errs, floors)]
    del pert, pert_out

    # CPU baseline (rank 0, N = 1 only): the oracle on a bounded, stratified
    # sample. Its results are also the parity check of the plain form: the
    # same bits as the reference's algorithm, matrix by matrix.
    cpu = None
    parity = None
    truth_check = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        oracle.lib()
        sample = cpu_sample(count, args.cpu_sample)
        t0 = time.perf_counter()
        refs = [oracle.expm(mats[i]) for i in sample]
        dt = time.perf_counter() - t0
        equal, decisions, worst = 0, 0, 0.0
        for i, (ref, info) in zip(sample, refs):
            got = plain["outs"][i].cpu().numpy().T
            equal += bool(np.array_equal(got, ref))
            d = plain["diags"][i]
            decisions += (d.degree, d.squarings) == (info["degree"], info["squarings"])
            worst = max(worst, float(np.abs(got - ref).sum(axis=0).max() / np.abs(ref).sum(axis=0).max()))
        omg = OMEGAS(count)
        sample_cost = sum(expm_cost(orders[i], plain["diags"][i].squarings) for i in sample)
        sweep_cost = sum(expm_cost(n, d.squarings) for n, d in zip(orders, plain["diags"]))
        desc = (f"stratified: {len(sample)} matrices, every {sample[1] - sample[0] if len(sample) > 1 else 1}-th of "
                f"this sweep (omega {omg[sample[0]]:.3g}..{omg[sample[-1]]:.3g}, orders "
                f"{[orders[i] for i in sample]}, squarings {[plain['diags'][i].squarings for i in sample]}), "
                f"{dt:.1f} s, C++ restatement of the reference, all host threads")
        cpu = {"value": len(sample) / dt, "unit": "expm/s", "cores": oracle.threads(), "kind": "port",
               "sample": desc, "sample_cost_n3_s8": sample_cost, "sweep_cost_n3_s8": sweep_cost,
               "cost_weighted_value": (sample_cost / dt) / (sweep_cost / count),
               "cost_weighted_note": "sample cost per second / mean sweep cost per matrix: the CPU rate had it "
                                     "run the whole sweep's mix"}
        parity = {"matrices_compared": len(sample), "bit_identical": equal, "decisions_equal": decisions,
                  "max_rel_err_1norm": worst}
        # Both forms against exp(A) itself (the extended-precision exponential),
        # on the sweep's smallest matrices, one per frequency band.
        from oracle.extended import expm_extended, has_extended_precision, rel1_extended
        if has_extended_precision():
            bands = np.array_split(np.arange(count), args.truth_sample)
            picks = [int(b[np.argmin([orders[i] for i in b])]) for b in bands if len(b)]
            rows = []
            for i in picks:
                truth = expm_extended(mats[i])
                rows.append({"n": orders[i], "squarings": plain["diags"][i].squarings,
                             "plain_vs_exact": rel1_extended(plain["outs"][i].cpu().numpy().T, truth),
                             "split_vs_exact": rel1_extended(split["outs"][i].cpu().numpy().T, truth)})
            truth_check = {"matrices": rows,
                           "max_split_over_plain": max(r["split_vs_exact"] / r["plain_vs_exact"] for r in rows),
                           "exact": "exp(A) by Taylor scaling and squaring in 80-bit long double (about 2^-9 of "
                                    "an FP64 computation's rounding on these matrices)"}

    def dmma_roofline(r):
        st = r["st"]
        achieved = st["gemm_flops"] / (st["gemm_ms"] * 1e-3) / 1e12 if st["gemm_ms"] > 0 else None
        return {"bound": "tensor", "kernel": "gemm_dmma_kernel (FP64 DMMA, complex 4M)",
                "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                "frac": (achieved / peak64) if (achieved and peak64) else None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this process (MEASURED_PEAKS.json has no FP64 figure)",
                "traffic": (GEMM_TRAFFIC_RATIO * st["gemm_bytes"] / st["gemm_launches"])
                           if st["gemm_launches"] else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum over every GEMM launch of "
                                  "the 16-matrix sweep = 0.711 x its algorithmic bytes, scaled to this sweep's "
                                  "algorithmic bytes per launch",
                "timing": "CUDA events around every GEMM launch of one extra sweep run as a single group",
                "gemm_launches_per_sweep": int(st["gemm_launches"]),
                "gemm_tflop_per_sweep": st["gemm_flops"] / 1e12,
                "algorithmic_bytes_per_launch": st["gemm_bytes"] / st["gemm_launches"] if st["gemm_launches"] else None}

    # matrices the whole job processed per step: every rank's share
    jobs = args.count * world if (args.shard == "lpt" and world > 1) else count * world
    def rate(ms):
        return jobs / (ms * 1e-3) if ms else None

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        del host_in, host_out
        configs = other_configurations(args, ws, torch, peak64, peak8, (orders, mats, dev_in))

    sst = split["st"]
    # Algorithmic int8 operations: per modulus, the real embedding of each
    # complex product (m x 2k times 2k x 2n), 8mnk, the same count as the
    # product's FP64 flops; the kernel issues more on the padded residue
    # extents (m to 128 rows, 2n to the tile width, 2k to 128).
    int8_tops = (args.moduli * sst["split_flops"] / (sst["split_ms"] * 1e-3) / 1e12
                 if sst["split_ms"] > 0 else None)
    issued_tops = sst["split_int8_ops"] / (sst["split_ms"] * 1e-3) / 1e12 if sst["split_ms"] > 0 else None
    degrees = sorted(set((d.degree, d.squarings) for d in split["diags"]))
    if rank == 0:
        line = {
            "metric": METRIC, "value": rate(split["ms"]), "unit": "expm/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": split["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": f"f64 results; Expm's products from int8 residues modulo {args.moduli} moduli "
                     "(exact int32 sums, CRT reconstruction in f64); decisions, LU and solve in f64",
            "data": "synthetic, seeded",
            "config": {"workload": WORKLOAD, "count": count, "seed": args.seed, "autotune": bool(args.autotune),
                       "form": f"split precision, {args.moduli} moduli (tcgen05 kind::i8, Chinese remainder "
                               "reconstruction) for every product of Expm (A^2, A^4, A^6 with bounds that settle the "
                               "reference's degree and s, else recomputed in FP64); norms, normest1, LU and the Pade "
                               "solve in plain FP64",
                       "l2": f"inputs larger than L2: {in_bytes / 1e9:.2f} GB of matrices per step per GPU",
                       "parallelism": f"independent matrices; {shard_note}",
                       "squarings_range": [min(s for _, s in degrees), max(s for _, s in degrees)]},
            "e2e": {"value": rate(split["e2e_ms"]), "unit": "expm/s", "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": in_bytes},
            "roofline": {"bound": "tensor", "kernel": "modular_gemm_kernel (tcgen05.mma kind::i8, TMEM accumulators)",
                         "achieved": int8_tops, "peak": peak8, "unit": "TOPS (int8)",
                         "frac": (int8_tops / peak8) if (int8_tops and peak8) else None,
                         "peak_source": peak8_src,
                         "fp64_equivalent_tflops": sst["split_flops"] / (sst["split_ms"] * 1e-3) / 1e12
                         if sst["split_ms"] > 0 else None,
                         "traffic": (SPLIT_TRAFFIC_RATIO * sst["split_bytes"] / sst["split_launches"])
                         if sst["split_launches"] else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum over every modular_gemm "
                                           "launch of the 16-matrix sweep = 1.044 x its algorithmic bytes, scaled to "
                                           "this sweep's algorithmic bytes per launch",
                         "timing": "CUDA events around every split-product launch of one extra sweep run as a "
                                   "single group; achieved counts the algorithmic int8 operations (moduli x 8mnk "
                                   "per complex product), achieved_issued those on the padded residue extents",
                         "achieved_issued": issued_tops,
                         "frac_issued": (issued_tops / peak8) if (issued_tops and peak8) else None,
                         "split_launches_per_sweep": int(sst["split_launches"]),
                         "split_int8_pops_per_sweep": args.moduli * sst["split_flops"] / 1e15,
                         "split_int8_pops_issued_per_sweep": sst["split_int8_ops"] / 1e15,
                         "algorithmic_bytes_per_launch": sst["split_bytes"] / sst["split_launches"]
                         if sst["split_launches"] else None},
            "split_accuracy": {
                "vs": "plain FP64 GPU form (bit-identical to the reference's CPU result)",
                "rel_err_1norm_max": max(errs), "rel_err_1norm_median": statistics.median(errs),
                "frac_within_1e-12": sum(e <= 1e-12 for e in errs) / len(errs),
                "max_ratio_to_fp64_floor": max(ratios), "median_ratio_to_fp64_floor": statistics.median(ratios),
                "fp64_floor": "per matrix, ||expm(A(1+2^-52 z)) - expm(A)||_1 / ||expm(A)||_1 in the plain form, "
                              "z ~ N(0,1) entrywise: the distance any arithmetic that is not the reference's bit "
                              "for bit can be expected to have",
                "fp64_floor_max": max(floors),
                "decisions": "degree and s equal the plain form's (the reference's) for every matrix (asserted); "
                             "A^2, A^4, A^6 from the split product with bounds holding the reference's d4, d6; "
                             "matrices whose decision was not settled on the bounds recomputed them in FP64",
                "exact_fallbacks_per_sweep": int(split["st"]["exact_fallbacks"]),
                "vs_exact": truth_check},
            "plain_fp64": {"value": rate(plain["ms"]), "ms_per_step": plain["ms"],
                           "e2e": rate(plain["e2e_ms"]), "gpu_launches": int(plain["st_step"]["kernel_launches"]),
                           "parity_vs_reference": parity, "roofline": dmma_roofline(plain),
                           "clocks": plain["clocks"]},
            "cpu_baseline": cpu,
            "configurations": configs,
            "clocks": split["clocks"],
            "gpu_launches": int(split["st_step"]["kernel_launches"]),
        }
        print(json.dumps(line), flush=True)
    ws.dispose()


def measured_hbm_peak():
    """The copy bandwidth (GB/s) MEASURED_PEAKS.json holds, else 6650 GB/s (an
    earlier copy-bandwidth measurement of a B200), with where it came from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        for k in ("hbm_gbs", "hbm_GBps", "hbm"):
            if isinstance(d.get(k), (int, float)):
                return float(d[k]), "MEASURED_PEAKS.json " + k
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback 6650 GB/s (an earlier B200 copy-bandwidth measurement)"


def other_configurations(args, ws, torch, peak64, peak8, sweep):
    """The other configurations of the workload, each measured once here, next
    to the CPU restatement of the reference on the same inputs (the oracle,
    all host threads) and its parity: the FP64 GEMM (1), the n = 512 dense
    path (2), the precision form of the solve at n = 4096 (3), the batched
    exponential action over the sweep (4, Expmv), and the differentiation
    form (5). GPU times are CUDA events on the library's stream around the
    public host-buffer call unless a field says otherwise, the median of a
    few runs with L2 flushed (a 256 MB write) before each."""
    from oracle import oracle
    oracle.lib()
    stream = torch.cuda.ExternalStream(ws.stream)
    flush_buf = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")  # 256 MB > L2

    def gpu_ms(fn, reps=3):
        times, out = [], None
        for _ in range(reps):
            flush_buf.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times), out

    def cpu_s(fn):
        t0 = time.perf_counter()
        out = fn()
        return time.perf_counter() - t0, out

    cores = oracle.threads()
    res = {}

    def wanted(k):
        return args.only_config in (0, k)

    # (1) FP64 GEMM m = n = k = 1024, uniform [-1, 1), alpha 1, beta 0.
    if wanted(1):
        config_gemm(args, ws, torch, oracle, res, gpu_ms, cpu_s, cores, peak64)
    if wanted(2):
        config_dense(args, ws, oracle, res, gpu_ms, cpu_s)
    if wanted(3):
        config_precision(args, ws, oracle, res, gpu_ms, cpu_s, peak8)
    if wanted(4):
        config_expmv(args, ws, torch, oracle, res, gpu_ms, cpu_s, sweep)
    if wanted(5):
        config_differentiation(args, ws, res, gpu_ms)
    return res


def config_gemm(args, ws, torch, oracle, res, gpu_ms, cpu_s, cores, peak64):
    """(1) FP64 GEMM m = n = k = 1024."""
    rng = np.random.default_rng(args.seed + 1)
    n = 1024
    a = np.asfortranarray(rng.uniform(-1.0, 1.0, (n, n)))
    b = np.asfortranarray(rng.uniform(-1.0, 1.0, (n, n)))
    da, db = torch.from_numpy(a.T.copy()).cuda(), torch.from_numpy(b.T.copy()).cuda()
    dc = torch.empty_like(da)
    dev_ms, _ = gpu_ms(lambda: ws._call("tns_dgemm_device", n, n, n, 1.0, da.data_ptr(), n, db.data_ptr(), n, 0.0,
                                        dc.data_ptr(), n), reps=5)
    e2e_ms, c = gpu_ms(lambda: ws.multiply(a, b), reps=5)
    cs, cref = cpu_s(lambda: oracle.gemm(a, b))
    cs1, _ = cpu_s(lambda: oracle.gemm(a, b, multithreaded=False))
    flops = 2.0 * n ** 3
    kernel_ms = []
    for _ in range(5):
        ws.reset_stats()
        ws.set_timing(True)
        ws._call("tns_dgemm_device", n, n, n, 1.0, da.data_ptr(), n, db.data_ptr(), n, 0.0, dc.data_ptr(), n)
        ws.set_timing(False)
        kernel_ms.append(ws.stats()["gemm_ms"])
    kms = statistics.median(kernel_ms)
    res["1_fp64_gemm_1024"] = {
        "value": flops / (dev_ms * 1e-3) / 1e9, "unit": "GFLOP/s", "ms": dev_ms,
        "timing": "tns_dgemm_device (operands in HBM, padded copies inside the call)",
        "e2e": {"value": flops / (e2e_ms * 1e-3) / 1e9, "unit": "GFLOP/s", "ms": e2e_ms,
                "h2d_bytes": 2 * 8 * n * n, "d2h_bytes": 8 * n * n},
        "roofline": {"bound": "tensor", "kernel": "gemm_dmma_kernel (FP64 DMMA)", "peak": peak64, "unit": "TFLOP/s",
                     "achieved": flops / (kms * 1e-3) / 1e12, "kernel_ms": kms,
                     "frac": (flops / (kms * 1e-3) / 1e12 / peak64) if peak64 else None,
                     "peak_source": "cuBLAS DGEMM 8192^3 in this process",
                     "timing": "CUDA events around the GEMM kernel alone (the call's padded copies leave the "
                               "operands in L2)"},
        "cpu_baseline": {"value": flops / cs / 1e9, "unit": "GFLOP/s", "cores": cores, "kind": "port",
                         "sample": "the same product, the reference's threaded blocking (KC 256)"},
        "cpu_baseline_one_thread": {"value": flops / cs1 / 1e9, "unit": "GFLOP/s", "cores": 1, "kind": "port",
                                    "sample": "the same product, the reference's serial Gemm (KC 384)"},
        "bit_identical_to_reference": bool(np.array_equal(c, cref))}
    del da, db, dc


def config_dense(args, ws, oracle, res, gpu_ms, cpu_s):
    """(2) n = 512: LU + solve of 8 right-hand sides + rcond, real and complex;
    Expm over 32 draws with ||A||_1 log-uniform in [1e-2, 1e3]."""
    n = 512
    two = {}
    for kind in ("real", "complex"):
        rng = np.random.default_rng(args.seed + (2 if kind == "real" else 3))
        if kind == "real":
            a = rng.standard_normal((n, n)) / math.sqrt(n)
            b = rng.standard_normal((n, 8))
        else:
            a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
            b = rng.standard_normal((n, 8)) + 1j * rng.standard_normal((n, 8))
        a = np.asfortranarray(a)

        def lu_path():
            lu = ws.factor_lu(a)
            return lu, lu.solve(b), lu.reciprocal_condition()

        ms_lu, (lu, x, rc) = gpu_ms(lu_path)
        cs_lu, (f, piv, _) = cpu_s(lambda: oracle.getrf(a))
        cs_s, xo = cpu_s(lambda: oracle.getrs(f, piv, b))
        cs_r, rco = cpu_s(lambda: oracle.gecon(f, piv, -1, oracle.norm1(a)))
        norms = np.exp(rng.uniform(math.log(1e-2), math.log(1e3), 32))
        draws = []
        for v in norms:
            g = rng.standard_normal((n, n)) / math.sqrt(n) if kind == "real" else \
                (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
            draws.append(np.asfortranarray(g * (v / np.abs(g).sum(axis=0).max())))
        from csharp_linearalgebra_b200 import ExpmDiagnostics
        diags = [ExpmDiagnostics() for _ in draws]
        outs = [None] * len(draws)

        def ladder():
            for q, d in enumerate(draws):
                outs[q] = ws.expm(d, diags[q])

        ms_ex, _ = gpu_ms(ladder, reps=1)
        cs_ex, refs = cpu_s(lambda: [oracle.expm(d) for d in draws])
        two[kind] = {
            "lu_solve8_rcond_ms": ms_lu,
            "lu_gflops": ((2.0 / 3.0) * n ** 3 * (4 if kind == "complex" else 1)) / (ms_lu * 1e-3) / 1e9,
            "cpu_lu_solve8_rcond_ms": 1e3 * (cs_lu + cs_s + cs_r),
            "pivots_equal": bool(np.array_equal(lu.pivots, piv)), "factors_equal": bool(np.array_equal(lu.factors, f)),
            "solution_equal": bool(np.array_equal(x, xo)), "rcond_equal": bool(rc == rco),
            "expm_ms_per_call": ms_ex / len(draws), "cpu_expm_ms_per_call": 1e3 * cs_ex / len(draws),
            "expm_decisions_equal": sum((d.degree, d.squarings) == (i["degree"], i["squarings"])
                                        for d, (_, i) in zip(diags, refs)),
            "expm_bit_identical": sum(bool(np.array_equal(o, r)) for o, (r, _) in zip(outs, refs)),
            "expm_draws": len(draws),
            "degrees_seen": sorted(set(d.degree for d in diags)),
            "squarings_range": [min(d.squarings for d in diags), max(d.squarings for d in diags)]}
    two["timing"] = ("GPU: the host-buffer calls (factor, solve, rcond; one Expm per draw, in sequence); "
                     "CPU: the oracle on all host threads, the same inputs")
    res["2_dense_path_512"] = two


def config_precision(args, ws, oracle, res, gpu_ms, cpu_s, peak8):
    """(3) precision form: n = 4096, 64 right-hand sides, A = U diag(sigma) V^T."""
    n, nrhs = 4096, 64
    rng = np.random.default_rng(args.seed + 4)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    b = np.asfortranarray(rng.standard_normal((n, nrhs)))
    three = {"kappa": {}}
    # one untimed call of each route first (module loading, memory pool)
    a0 = np.asfortranarray((u * np.logspace(0.0, -2.0, n)) @ v.T)
    ws.solve_mixed(a0, b)
    ws.factor_lu(a0).solve(b)
    del a0
    for kappa in (1e2, 1e6, 1e10):
        sig = np.logspace(0.0, -math.log10(kappa), n)
        a = np.asfortranarray((u * sig) @ v.T)
        ms_mx, (x, info) = gpu_ms(lambda: ws.solve_mixed(a, b), reps=3)

        def fp64():
            return ws.factor_lu(a).solve(b)

        ms_64, x64 = gpu_ms(fp64, reps=3)
        anorm = np.abs(a).sum(axis=1).max()

        def backward(xx):
            r = b - a @ xx
            return float(max(np.abs(r[:, j]).max() / (anorm * np.abs(xx[:, j]).max() + np.abs(b[:, j]).max())
                             for j in range(nrhs)))

        entry = {"mixed_ms": ms_mx, "fp64_ms": ms_64, "moduli": info["moduli"],
                 "factorizations": info["factorizations"], "refinement_steps": info["iterations"],
                 "route": "partial pivoting" if info["pivoting"] else "butterfly transforms, no pivoting",
                 "rcond_estimate": info["rcond"],
                 "backward_error_mixed": backward(x), "backward_error_fp64": backward(x64),
                 "rel_diff_mixed_vs_fp64": float(np.linalg.norm(x - x64) / np.linalg.norm(x64))}
        if kappa == 1e2:
            cs_f, (f, piv, _) = cpu_s(lambda: oracle.getrf(a))
            cs_s, xo = cpu_s(lambda: oracle.getrs(f, piv, b))
            entry["cpu_fp64_lu_solve_ms"] = 1e3 * (cs_f + cs_s)
            entry["fp64_bit_identical_to_reference"] = bool(np.array_equal(x64, xo))
            # One more FP64 factorization with per-phase CUDA events
            # (LuPhaseTimings' split), outside the timed calls above.
            ws.reset_stats()
            ws.set_lu_timing(True)
            ws.factor_lu(a)
            ws.set_lu_timing(False)
            entry["fp64_lu_phases_ms"] = ws.lu_timings()
        three["kappa"][f"{kappa:.0e}"] = entry
    ws.reset_stats()
    ws.set_timing(True)
    g1 = rng.uniform(-1.0, 1.0, (n, n))
    g2 = rng.uniform(-1.0, 1.0, (n, n))
    ws.multiply_split(g1, g2, args.moduli)
    ws.set_timing(False)
    st = ws.stats()
    three["split_gemm_4096"] = {
        "moduli": args.moduli, "kernel_ms": st["split_ms"],
        "fp64_equivalent_tflops": st["split_flops"] / (st["split_ms"] * 1e-3) / 1e12 if st["split_ms"] else None,
        "int8_tops": st["split_int8_ops"] / (st["split_ms"] * 1e-3) / 1e12 if st["split_ms"] else None,
        "int8_peak_tops": peak8,
        "timing": "CUDA events around the modular GEMM launches of one real 4096^3 split product"}
    three["timing"] = ("GPU: the host-buffer calls (factorization included), median of 3 after one untimed call "
                       "of each route; CPU: the oracle")
    res["3_precision_solve_4096"] = three


def config_expmv(args, ws, torch, oracle, res, gpu_ms, cpu_s, sweep):
    """(4) the batched exponential action over the benchmark's own sweep (on
    the device already): B n x 8, t = 0.5."""
    orders, all_mats, dev_a = sweep
    omegas = np.logspace(2.0, 6.0, len(orders))
    ms_sel, sel = gpu_ms(lambda: ws.expmv_select_batched([t.data_ptr() for t in dev_a], 8, 0.5, device=True,
                                                          orders=orders, lds=orders), reps=1)
    sub = [k for k in range(len(orders)) if omegas[k] <= args.expmv_wmax]
    rng = np.random.default_rng(args.seed + 5)
    bs = [np.asfortranarray(rng.standard_normal((orders[k], 8)) + 1j * rng.standard_normal((orders[k], 8)))
          for k in sub]
    dev_b = [torch.from_numpy(x.T.copy()).cuda() for x in bs]
    dev_o = [torch.empty_like(x) for x in dev_b]
    so = [orders[k] for k in sub]
    ms_dev, diags = gpu_ms(lambda: ws.expmv_batched_device(len(sub), so, [dev_a[k].data_ptr() for k in sub], so, 8,
                                                           [x.data_ptr() for x in dev_b], so, 0.5,
                                                           [x.data_ptr() for x in dev_o], so), reps=2)
    ms_e2e, outs = gpu_ms(lambda: ws.expmv_batched([all_mats[k] for k in sub], bs, 0.5), reps=1)
    apps = [d.applications for d in diags]
    abytes = sum(ap * 16.0 * nn * nn for ap, nn in zip(apps, so))
    fp64_instr = sum(ap * 64.0 * nn * nn for ap, nn in zip(apps, so))
    hbm_peak, hbm_src = measured_hbm_peak()
    cpu_pick = sub[:3]
    cs_mv, refs = cpu_s(lambda: [oracle.expmv(all_mats[k], bs[sub.index(k)], 0.5) for k in cpu_pick])
    res["4_batched_expmv"] = {
        "value": len(sub) / (ms_dev * 1e-3), "unit": "expmv/s", "ms": ms_dev,
        "matrices": len(sub), "omega_max": args.expmv_wmax,
        "subset": f"the sweep's matrices with w <= {args.expmv_wmax:g} ({len(sub)} of {len(orders)}); "
                  "above it the applications (about 1.4 w per matrix) grow past a benchmark step",
        "applications": sum(apps), "early_exits": sum(d.early_exits for d in diags),
        "e2e": {"value": len(sub) / (ms_e2e * 1e-3), "unit": "expmv/s", "ms": ms_e2e,
                "h2d_bytes": sum(16 * nn * nn + 16 * nn * 8 for nn in so), "d2h_bytes": sum(16 * nn * 8 for nn in so)},
        "roofline": {"bound": "fp64 pipe (exact-order products: a multiply and an add per term, no FMA)",
                     "kernel": "taylor_kernel (one cooperative launch)",
                     "achieved_a_bytes_gbs": abytes / (ms_dev * 1e-3) / 1e9, "hbm_peak_gbs": hbm_peak,
                     "hbm_frac": abytes / (ms_dev * 1e-3) / 1e9 / hbm_peak, "hbm_peak_source": hbm_src,
                     "achieved_fp64_tops": fp64_instr / (ms_dev * 1e-3) / 1e12,
                     "fp64_peak_tops_nominal": 148 * 64 * 1.965e9 / 1e12,
                     "fp64_frac": fp64_instr / (ms_dev * 1e-3) / (148 * 64 * 1.965e9),
                     "algorithmic_work": "per application 16 n^2 bytes of A and 64 n^2 FP64 operations "
                                         "(8 columns, 4 multiplies and 4 adds per complex term)"},
        "selection_all_256": {"ms": ms_sel, "sum_m_s": int(sum(m * s_ for m, s_ in sel)),
                              "sum_m_s_subset": int(sum(sel[k][0] * sel[k][1] for k in sub)),
                              "max_s": int(max(s_ for _, s_ in sel))},
        "cpu_baseline": {"value": len(cpu_pick) / cs_mv, "unit": "expmv/s", "cores": 1, "kind": "port",
                         "sample": f"the {len(cpu_pick)} lowest-frequency matrices of the subset (orders "
                                   f"{[orders[k] for k in cpu_pick]}), the oracle's sequential Expmv"},
        "parity": {"compared": len(cpu_pick),
                   "bit_identical": sum(bool(np.array_equal(outs[sub.index(k)], r)) for k, (r, _) in
                                        zip(cpu_pick, refs)),
                   "decisions_and_counts_equal": sum(
                       (diags[sub.index(k)].degree, diags[sub.index(k)].scaling, diags[sub.index(k)].applications)
                       == (i["degree"], i["scaling"], i["applications"]) for k, (_, i) in zip(cpu_pick, refs))}}
    del dev_b, dev_o


def config_differentiation(args, ws, res, gpu_ms):
    """(5) differentiation: gradient of ||exp(tA)B - Y||_F^2 at n = 2048
    (w = 1e4, B 2048 x 16, t = 1) and the Frechet derivative at n = 1024."""
    five = {}
    n = 2048
    a5 = sweep_matrix(10_000, n, 1e4, args.seed + 6)
    rng = np.random.default_rng(args.seed + 7)
    b5 = np.asfortranarray(rng.standard_normal((n, 16)) + 0j)
    y5 = np.asfortranarray(rng.standard_normal((n, 16)) + 1j * rng.standard_normal((n, 16)))
    ms_g, g = gpu_ms(lambda: ws.expmv_gradient(a5, b5, y5, 1.0), reps=1)
    from csharp_linearalgebra_b200 import ExpmvDiagnostics
    dv = ExpmvDiagnostics()
    ms_v, fv = gpu_ms(lambda: ws.expmv(a5, b5, 1.0, dv), reps=1)
    five["gradient_2048"] = {"ms": ms_g, "degree": g["degree"], "squarings": g["squarings"],
                             "f_vs_expmv_rel": float(np.linalg.norm(g["f"] - fv) / np.linalg.norm(fv))}
    five["expmv_2048x16"] = {"ms": ms_v, "degree": dv.degree, "scaling": dv.scaling,
                             "applications": dv.applications,
                             "a_bytes_gbs": dv.applications * 16.0 * n * n / (ms_v * 1e-3) / 1e9}
    n = 1024
    a6 = sweep_matrix(10_001, n, 1e4, args.seed + 8)
    e6 = np.asfortranarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ms_f, (x6, l6) = gpu_ms(lambda: ws.expm_frechet(a6, e6), reps=1)
    block = np.zeros((2 * n, 2 * n), dtype=np.complex128, order="F")
    block[:n, :n] = a6
    block[:n, n:] = e6
    block[n:, n:] = a6
    ms_b, eb = gpu_ms(lambda: ws.expm(block), reps=1)
    five["frechet_1024"] = {
        "ms": ms_f, "block_expm_2048_ms": ms_b,
        "rel_diff_vs_block_expm": float(np.abs(l6 - eb[:n, n:]).sum(axis=0).max() / np.abs(eb[:n, n:]).sum(axis=0).max()),
        "block_expm": "the reference's route, Expm of [[A, E], [0, A]], in this library's plain form (the "
                      "reference's arithmetic bit for bit)"}
    five["cpu_baseline"] = None
    five["cpu_baseline_note"] = ("not timed by default: the reference's route is Expm of the 2048-order block, "
                                 "tens of seconds of the oracle")
    res["5_differentiation"] = five


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--count", type=int, default=256)
    p.add_argument("--groups", type=int, default=4, help="cost-balanced groups run concurrently")
    p.add_argument("--seed", type=int, default=20260915)
    p.add_argument("--cpu-sample", type=int, default=16, help="matrices in the stratified CPU sample")
    p.add_argument("--ref-chunks", type=int, default=4, help="reference arm: the sample in this many steps")
    p.add_argument("--truth-sample", type=int, default=8, help="matrices checked against the extended-precision exp")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    p.add_argument("--no-peak", action="store_true", help="skip the measured FP64/INT8 peaks (profiling runs)")
    # 17 moduli: t = 59 integer bits for K' <= 2048, so each split product's own error (about K' 2^-t of
    # its scales) is near the FP64 unit roundoff. Measured on this sweep, the distance to the reference
    # and to exp(A) itself is that of 18 or 20 moduli (it is set by the FP64 steps' rounding): at most
    # 4.50 floors from the reference with 17 moduli, 4.46 with 18; 16 moduli measured 5.12.
    p.add_argument("--moduli", type=int, default=17, help="moduli of the split-precision form (8..22)")
    p.add_argument("--autotune", type=int, default=0, help="1: GEMM launch shapes chosen by timing (tns_set_autotune)")
    p.add_argument("--no-configs", action="store_true", help="skip the other configurations' measurements")
    p.add_argument("--configs-only", action="store_true", help="only the other configurations' measurements")
    p.add_argument("--only-config", type=int, default=0, help="with --configs-only: just this one (1..5)")
    p.add_argument("--expmv-wmax", type=float, default=1e4,
                   help="batched Expmv: time the sweep's matrices up to this frequency")
    p.add_argument("--shard", choices=["lpt", "seeds"], default="lpt",
                   help="N > 1: one LPT-partitioned sweep (lpt) or a sweep per rank (seeds)")
    args = p.parse_args()
    world, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            ours(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
