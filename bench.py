"""Benchmarks of the exact-SRE / MC_SRE / Mana hot path on B200, one configuration per run.

    python bench.py [--config c2] [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    torchrun --nnodes=1 --nproc-per-node N --master-addr 127.0.0.1 bench.py --gpus N
    python bench.py --profile-case --n 20 --k0 1024 --count 256 --precision fp64

Configurations (synthetic seeded inputs: numpy default_rng, real and imaginary parts
N(0, 1), normalised; the reference publishes no benchmark input):

  c2 (default)  exact SRE q=2, N=20 (seed 20), FP64: one step = all 2^20 X-strings x
                2^20-point transforms = 4^20 Pauli strings
  c2fp32        the same with FP32 butterflies and FP64 powers / sums
  c2q3          q = 2 and 3 from one sweep, N=20, FP64 (--precision fp32 for FP32)
  c1            exact SRE q=2, N=12 (seed 12), FP64
  c2mc          MC_SRE q=2 on the N=20 state: 13 beta chains x 76,924 steps = 1.0e6
                Metropolis proposals, injected proposal stream (seed 123)
  c3            batched exact SRE: 512 states, N_i ~ U{8..18} (seed 512), states seed
                10000+i, q in {2, 3}, FP32 (--precision fp64 for FP64); compared with
                per-state hm_sre calls and with the plain GPU form (HM_PLAIN)
  c4n14, c4n18  adjoint dSRE_2/dpsi at N = 14 / 18 (seeds 14 / 18), FP64; compared with
                the forward sweep of the same state
  c5pure        Mana of a 10-qutrit pure state (seed 10)
  c5mixed       Mana of the 729 x 729 density matrix of that state traced over its 4
                least significant qutrits

Every run prints one JSON line on rank 0: `value` = the metric of the whole job with the
inputs resident in device memory (CUDA events on the library's stream, L2 flushed by a
256 MiB write before every step, max over ranks), `e2e` = the same metric through the C
ABI call with host buffers (host-device copies inside the timed region), `roofline` =
the dominant kernel's algorithmic work against the device's measured FP64 rate (DADD
probe) or HBM copy bandwidth, `cpu_baseline` = the oracle (a C restatement of the
reference's :threads backend) on a bounded sample with all host threads.
`--impl reference` times that CPU restatement alone on the same workload (the reference
itself is Julia, which this image does not ship).  `--profile-case` runs a short
hm_sre_range / hm_sre_grad / Mana workload for ncu and prints its sums.
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
sys.path.insert(0, ROOT)

FLUSH_BYTES = 256 << 20  # larger than the 126 MB L2

CONFIGS = {
    "c1": dict(kind="sre", n=12, seed=12, qs=(2.0,), precision="fp64"),
    "c2": dict(kind="sre", n=20, seed=20, qs=(2.0,), precision="fp64"),
    "c2fp32": dict(kind="sre", n=20, seed=20, qs=(2.0,), precision="fp32"),
    "c2q3": dict(kind="sre", n=20, seed=20, qs=(2.0, 3.0), precision="fp64"),
    "c2mc": dict(kind="mc", n=20, seed=20, nbeta=13, nsamples=76924, stream_seed=123),
    "c3": dict(kind="batched", nstates=512, nmin=8, nmax=18, count_seed=512, qs=(2.0, 3.0), precision="fp32"),
    "c4n14": dict(kind="grad", n=14, seed=14),
    "c4n18": dict(kind="grad", n=18, seed=18),
    "c5pure": dict(kind="mana_pure", L=10, seed=10),
    "c5mixed": dict(kind="mana_mixed", L=10, seed=10, keep=6),
}


# default timed steps: about a second of timed work or more per configuration, so that
# the clock sampler (200 ms period) sees the timed region
DEFAULT_STEPS = {"c1": 200, "c4n14": 300, "c5pure": 40, "c5mixed": 400}


def make_state(dim, seed):
    g = np.random.default_rng(seed)
    v = g.normal(size=dim) + 1j * g.normal(size=dim)
    return v / np.linalg.norm(v)


def batched_states(cfg):
    counts = np.random.default_rng(cfg["count_seed"]).integers(cfg["nmin"], cfg["nmax"] + 1, size=cfg["nstates"])
    ns = [int(v) for v in counts]
    return ns, [make_state(1 << n, 10_000 + i) for i, n in enumerate(ns)]


def fp64_ops_per_x(n, nq=1):
    """FP64-pipe operations of one X-string: n 2^n butterfly adds, 2 2^n for the product
    f = conj(psi(r)) psi(r ^ x), 4 2^n for the q = 2 moments (one more mul and fma per
    value for each further q in {3})."""
    return (n + 6 + 2 * (nq - 1)) * (1 << n)


def physical_cores():
    try:
        import psutil
        return psutil.cpu_count(logical=False) or os.cpu_count()
    except Exception:
        return os.cpu_count()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler is producing samples
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "samples": len(sm),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------ CPU side

def _oracle():
    from oracle import oracle as O
    O.build()
    return O


def cpu_sre_sample(n, seed, qs, seconds):
    """Oracle fast path (or_sre_sums_fast: build + FWHT + moments of src/SRE.jl:338-540 on
    the static partition of src/Backends/Threads.jl:37-102) over the first k X-strings of
    every thread's slice of the whole Gray range, k sized for about `seconds`; returns
    Pauli strings / s over all 4^n of one X-string's worth per X-string."""
    O = _oracle()
    psi = make_state(1 << n, seed)
    threads = os.cpu_count() or 1
    dim = 1 << n
    O.sre_sums_fast(psi, qs, 1, dim, nthreads=threads, per_thread=1)  # thread start-up, first touch
    t = time.perf_counter()
    O.sre_sums_fast(psi, qs, 1, dim, nthreads=threads, per_thread=2)
    dt = max(time.perf_counter() - t, 1e-4)
    per = int(max(1, min(dim // threads, seconds / dt * 2)))
    t = time.perf_counter()
    O.sre_sums_fast(psi, qs, 1, dim, nthreads=threads, per_thread=per)
    dt = time.perf_counter() - t
    count = per * min(threads, dim)
    return {"value": count * float(dim) / dt, "unit": "Pauli-strings/s", "cores": threads,
            "physical_cores": physical_cores(), "kind": "port",
            "sample": f"{count} X-strings: the first {per} Gray indices of each of the {threads} threads' "
                      f"static slices of the N={n} sweep (q = {list(qs)}), {dt:.1f} s; oracle/hm_oracle.c "
                      f"or_sre_sums_fast (AVX2, OpenMP), extrapolated to the whole sweep at the same rate"}


def cpu_mc_sample(n, seed, nbeta, steps_per_chain, stream_seed):
    import hadamag_b200 as hm
    O = _oracle()
    psi = make_state(1 << n, seed)
    pd, rs = hm.proposal_stream(n, nbeta, steps_per_chain, seed=stream_seed)
    t = time.perf_counter()
    O.mc_sre(psi, 2, nbeta, steps_per_chain, pd, rs, nthreads=os.cpu_count())
    dt = time.perf_counter() - t
    props = nbeta * steps_per_chain
    return {"value": props * float(1 << n) / dt, "unit": "Pauli-strings/s", "cores": min(nbeta, os.cpu_count()),
            "physical_cores": physical_cores(), "kind": "port",
            "sample": f"{nbeta} chains x {steps_per_chain} steps ({props} proposals) of the N={n} chain, "
                      f"{dt:.1f} s, one chain per thread as src/Backends/Threads.jl:192 (oracle or_mc_sre)"}


def cpu_batched_sample(ns, psis, qs, seconds):
    O = _oracle()
    threads = os.cpu_count() or 1
    order = np.random.default_rng(7).permutation(len(ns))
    done, work, t0 = 0, 0.0, time.perf_counter()
    for i in order:
        n = ns[i]
        O.sre_sums_fast(psis[i], qs, 1, 1 << n, nthreads=threads)
        done += 1
        work += 4.0 ** n * len(qs)
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": work / dt, "unit": "Pauli-strings*q/s", "cores": threads, "physical_cores": physical_cores(),
            "kind": "port", "sample": f"{done} of the {len(ns)} states in a seeded random order, every X-string, "
                                      f"{dt:.1f} s (oracle or_sre_sums_fast)"}


def cpu_grad(n, seed):
    O = _oracle()
    psi = make_state(1 << n, seed)
    m = min(n, 14)
    p = make_state(1 << m, seed)
    t = time.perf_counter()
    O.sre_grad(p, 2)
    dt = time.perf_counter() - t
    rate = 4.0 ** m / dt
    del psi
    note = "" if m == n else f"; measured at N={m}, the N={n} rate assumed equal per Pauli string"
    return {"value": rate, "unit": "Pauli-strings/s", "cores": os.cpu_count(), "physical_cores": physical_cores(),
            "kind": "port", "sample": f"full gradient at N={m}, {dt:.1f} s (oracle or_sre_grad){note}"}


def cpu_mana_pure(L, seed, seconds):
    O = _oracle()
    psi = make_state(3 ** L, seed)
    dim = 3 ** L
    t = time.perf_counter()
    O.mana_sum(psi, 1, 64)
    dt = max(time.perf_counter() - t, 1e-4)
    cnt = int(min(dim, max(64, seconds / dt * 64)))
    t = time.perf_counter()
    O.mana_sum(psi, 1, cnt)
    dt = time.perf_counter() - t
    return {"value": cnt * float(dim) / dt, "unit": "phase-points/s", "cores": os.cpu_count(),
            "physical_cores": physical_cores(), "kind": "port",
            "sample": f"{cnt} of the {dim} ternary X-strings, {dt:.1f} s (oracle or_mana_sum)"}


def cpu_mana_mixed(rho):
    O = _oracle()
    t = time.perf_counter()
    O.mana_mixed(rho)
    dt = time.perf_counter() - t
    dim = rho.shape[0]
    return {"value": dim * dim / dt, "unit": "phase-points/s", "cores": 1, "physical_cores": physical_cores(),
            "kind": "port", "sample": f"the full {dim}x{dim} matrix, {dt * 1e3:.1f} ms (oracle or_mana_mixed)"}


# ------------------------------------------------------------------------------ GPU side

class Gpu:
    """The library context on this rank's GPU, its stream, an L2 flush buffer and event
    timing on that stream."""

    def __init__(self, local):
        import torch
        import hadamag_b200 as hm
        self.torch, self.hm = torch, hm
        torch.cuda.set_device(local)
        self.dev = torch.device("cuda", local)
        self.ctx = hm._native.Context(local)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.ctx.set_stream(self.stream.cuda_stream)
        self.flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=self.dev)

    def timed(self, fn):
        """Flush L2, run fn() between two events on the library stream; returns
        (fn's result, elapsed ms)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            self.flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
        r = fn()
        with torch.cuda.stream(self.stream):
            e1.record(self.stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    def upload(self, psi):
        return self.torch.from_numpy(np.ascontiguousarray(psi).view(np.float64).copy()).to(self.dev)


def run_steps(args, gpu, step, world, dist):
    """W untimed steps, then K timed steps between barriers; step() returns (ms, kernels)."""
    def barrier():
        if world > 1:
            dist.barrier()
        gpu.torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    times, launches = [], 0
    with ClockSampler(gpu.dev.index) as clk:
        barrier()
        for _ in range(args.steps):
            ms, nl = step()
            times.append(ms)
            launches += nl
        barrier()
    total = float(np.sum(times))
    if world > 1:
        t = gpu.torch.tensor([total], dtype=gpu.torch.float64, device=gpu.dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    return total, launches, clk.summary()


def roofline_fp64(ops, ms, peak, note):
    achieved = ops / (ms * 1e-3)
    return {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Top/s (FP64 pipe)",
            "frac": achieved / peak, "traffic": None,
            "peak_source": "measured live on this GPU: register-resident DADD kernel (hm_probe_fp64_peak)",
            "work": note}


def fp32_path_ops(n, nq):
    """FP32-butterfly path, per X-string: (n + 2) 2^n FP32 ops (butterflies and the FP32
    build of f) and (4 + 2 (nq - 1)) 2^n FP64 ops (the moment sums)."""
    return float((n + 2) * (1 << n)), float((4 + 2 * (nq - 1)) * (1 << n))


def roofline_fp32(ops32, ops64, ms, peak32, peak64):
    """FP32 ops against the FP32 add peak, FP64 ops against the FP64 add peak; the pipe
    whose work takes longer at its peak is the bound and gives the fraction."""
    t32, t64 = ops32 / peak32, ops64 / peak64
    f32, f64 = (ops32 / (ms * 1e-3)) / peak32, (ops64 / (ms * 1e-3)) / peak64
    if t32 >= t64:
        return {"bound": "fp32", "achieved": ops32 / (ms * 1e-3) / 1e12, "peak": peak32 / 1e12,
                "unit": "Top/s (FP32 pipe)", "frac": f32, "traffic": None,
                "peak_source": "measured live on this GPU: register-resident FADD kernel (hm_probe_fp32_peak)",
                "work": "(n + 2) 2^n FP32 ops per X-string (butterflies, build); the FP64 moment sums "
                        "(4 + 2 (nq - 1)) 2^n take less time at their peak",
                "fp64_pipe_frac": f64}
    return {"bound": "fp64", "achieved": ops64 / (ms * 1e-3) / 1e12, "peak": peak64 / 1e12,
            "unit": "Top/s (FP64 pipe)", "frac": f64, "traffic": None,
            "peak_source": "measured live on this GPU: register-resident DADD kernel (hm_probe_fp64_peak)",
            "work": "(4 + 2 (nq - 1)) 2^n FP64 moment ops per X-string; the FP32 butterflies take less time",
            "fp32_pipe_frac": f32}


def base_line(args, cfg_name, metric, unit, value, world, total_ms, dtype, workload, extra_cfg):
    return {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic: seeded complex-Gaussian states (numpy default_rng), normalised",
        "config": dict({"name": cfg_name, "workload": workload,
                        "l2": "flushed before every step (256 MiB write)"}, **extra_cfg),
    }


def fixture_check(n, seed, qs, precision, p2, m):
    """Compare the step's double-double sums with the committed oracle fixture."""
    path = os.path.join(ROOT, "tests", "golden", f"n{n}_seed{seed}.json")
    if not os.path.exists(path):
        return None
    fx = json.load(open(path))
    dim = float(1 << n)
    out = {"fixture": os.path.relpath(path, ROOT)}
    for i, q in enumerate(qs):
        if q in fx["qs"]:
            j = fx["qs"].index(q)
            ref = fx["sre"][j]
            val = float(-np.log2((m[i, 0] + m[i, 1]) / dim))
            out[f"sre_q{q:g}"] = val
            out[f"oracle_q{q:g}"] = ref
            out[f"rel_err_q{q:g}"] = abs(val / ref - 1.0)
    out["tolerance"] = 1e-10 if precision == "fp64" else 1e-6
    return out


def bench_sre(args, cfg, gpu, world, rank, dist):
    hm = gpu.hm
    from hadamag_b200 import shard
    n, qs = cfg["n"], cfg["qs"]
    precision = args.precision or cfg["precision"]
    prec = hm.PRECISIONS[precision]
    psi_host = make_state(1 << n, cfg["seed"])
    psi_dev = gpu.upload(psi_host)
    kb, ke = shard.gray_slice(n, rank, world)
    last = {}

    def step():
        (p2, m), ms = gpu.timed(lambda: gpu.ctx.sre_range_dev(psi_dev.data_ptr(), n, kb, ke, qs, prec))
        last["p"] = np.concatenate([p2, m.reshape(-1)])
        return ms, gpu.ctx.last_launch_count()

    total_ms, launches, clocks = run_steps(args, gpu, step, world, dist)
    gathered = shard.allgather_partials(last["p"], device=gpu.dev) if world > 1 else last["p"][None, :]
    sre, lost = shard.combine_partials(gathered, n, len(qs))
    folded = shard.dd_fold_rows(gathered)
    units = 4.0 ** n
    value = units * args.steps / (total_ms * 1e-3)

    def e2e_step():
        _, ms = gpu.timed(lambda: gpu.ctx.sre_range(psi_host, kb, ke, qs, prec))
        return ms, 0

    e2e_ms, _, _ = run_steps(argparse.Namespace(warmup=1, steps=args.steps), gpu, e2e_step, world, dist)
    my_ms = total_ms / args.steps
    if precision == "fp32":
        o32, o64 = fp32_path_ops(n, len(qs))
        nx = float(ke - kb)
        roof = roofline_fp32(o32 * nx, o64 * nx, my_ms, gpu.ctx.probe_fp32_peak(), gpu.ctx.probe_fp64_peak())
    else:
        ops = fp64_ops_per_x(n, len(qs)) * float(ke - kb)
        roof = roofline_fp64(ops, my_ms, gpu.ctx.probe_fp64_peak(),
                             f"(n + 6 + 2 (nq - 1)) 2^n FP64 ops per X-string x {ke - kb} X-strings per step")
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(prof) and precision in json.load(open(prof)) and n == 20:
        d = json.load(open(prof))[precision]
        roof["traffic"] = d["dram_bytes_per_x"] * float(ke - kb)
        roof["traffic_unit"] = "DRAM bytes (read + write) per step of this rank"
        roof["traffic_note"] = d["note"]
    qtxt = ",".join(f"{q:g}" for q in qs)
    line = base_line(args, args.config, f"Pauli-strings/s for exact SRE q={qtxt} N={n}", "Pauli-strings/s",
                     value, world, total_ms,
                     "f64" if precision == "fp64" else "f32-butterflies/f64-reduction",
                     f"exact SRE q={qtxt}, N={n}: 2^{n} X-strings x 2^{n}-point WHT = 4^{n} Pauli strings per step",
                     {"n": n, "q": list(qs), "precision": precision, "seed": cfg["seed"], "engine": args.engine,
                      "parallelism": f"gray-range split x{world}", "sre": [float(v) for v in sre],
                      "lost_norm": float(lost)})
    line["roofline"] = roof
    line["e2e"] = {"value": units * args.steps / (e2e_ms * 1e-3), "unit": "Pauli-strings/s",
                   "h2d_bytes_per_step": int(world * 16 * (1 << n)), "d2h_bytes_per_step": int(world * 8 * 2 * (1 + len(qs)))}
    line["gpu_launches"] = int(launches)
    line["clocks"] = clocks
    fx = fixture_check(n, cfg["seed"], qs, precision, folded[:2], folded[2:].reshape(len(qs), 2))
    if fx:
        line["parity"] = fx
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sre_sample(n, cfg["seed"], qs, 12.0)
    return line


def bench_mc(args, cfg, gpu, world, rank, dist):
    hm = gpu.hm
    from hadamag_b200 import shard
    n, nb, ns = cfg["n"], cfg["nbeta"], cfg["nsamples"]
    psi = make_state(1 << n, cfg["seed"])
    pd, rs = hm.proposal_stream(n, nb, ns, seed=cfg["stream_seed"])
    cb, ce = shard.chain_slice(nb, rank, world)
    res = {}

    def step():
        def call():
            res["r"] = gpu.ctx.mc_sre_chains(psi, 2.0, nb, cb, ce, ns, pd[cb:ce], rs[cb:ce])
        _, ms = gpu.timed(call)
        return gpu.ctx.last_kernel_ms(), gpu.ctx.last_launch_count()

    total_ms, launches, clocks = run_steps(args, gpu, step, world, dist)
    props = nb * ns
    units = props * float(1 << n)
    value = units * args.steps / (total_ms * 1e-3)

    def e2e_step():
        _, ms = gpu.timed(lambda: gpu.ctx.mc_sre_chains(psi, 2.0, nb, cb, ce, ns, pd[cb:ce], rs[cb:ce]))
        return ms, 0

    e2e_ms, _, _ = run_steps(argparse.Namespace(warmup=1, steps=args.steps), gpu, e2e_step, world, dist)
    m2 = None
    if world == 1:
        m2 = float(gpu.ctx.mc_sre(psi, 2.0, nb, ns, pd, rs)[0])
    ops = fp64_ops_per_x(n) * float((ce - cb) * ns)
    line = base_line(args, args.config, f"Pauli-strings/s for MC_SRE q=2 N={n} ({props} proposals)",
                     "Pauli-strings/s", value, world, total_ms, "f64",
                     f"MC_SRE q=2, N={n}: {nb} beta chains x {ns} Metropolis steps, each step one 2^{n}-point "
                     f"transform per chain ({props} proposals x 2^{n} Pauli strings per step)",
                     {"n": n, "nbeta": nb, "nsamples": ns, "stream_seed": cfg["stream_seed"],
                      "parallelism": f"beta-chain split x{world}", "m2": m2})
    line["roofline"] = roofline_fp64(ops, total_ms / args.steps, gpu.ctx.probe_fp64_peak(),
                                     "(n + 6) 2^n FP64 ops per proposal")
    line["e2e"] = {"value": units * args.steps / (e2e_ms * 1e-3), "unit": "Pauli-strings/s",
                   "h2d_bytes_per_step": int(16 * (1 << n) + 16 * props), "d2h_bytes_per_step": int(32 * nb)}
    line["gpu_launches"] = int(launches)
    line["clocks"] = clocks
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_mc_sample(n, cfg["seed"], nb, 40, cfg["stream_seed"])
    return line


def bench_batched(args, cfg, gpu, world, rank, dist):
    hm = gpu.hm
    from hadamag_b200 import shard
    precision = args.precision or cfg["precision"]
    prec = hm.PRECISIONS[precision]
    qs = cfg["qs"]
    ns, psis = batched_states(cfg)
    mine = shard.balance_states(ns, world)[rank]
    my_ns = [ns[i] for i in mine]
    my_psis = [psis[i] for i in mine]
    units_mine = sum(4.0 ** n for n in my_ns) * len(qs)
    units_all = sum(4.0 ** n for n in ns) * len(qs)

    def step():
        _, ms = gpu.timed(lambda: gpu.ctx.sre_batched(my_psis, qs, prec))
        return gpu.ctx.last_kernel_ms(), gpu.ctx.last_launch_count()

    total_ms, launches, clocks = run_steps(args, gpu, step, world, dist)
    value = units_all * args.steps / (total_ms * 1e-3)

    def e2e_step():
        _, ms = gpu.timed(lambda: gpu.ctx.sre_batched(my_psis, qs, prec))
        return ms, 0

    e2e_ms, _, _ = run_steps(argparse.Namespace(warmup=1, steps=args.steps), gpu, e2e_step, world, dist)
    line = base_line(args, args.config, "Pauli-strings*q/s for batched exact SRE (512 states, N 8..18, q 2,3)",
                     "Pauli-strings*q/s", value, world, total_ms,
                     "f64" if precision == "fp64" else "f32-butterflies/f64-reduction",
                     "batched exact SRE: 512 states, N_i ~ U{8..18} (seed 512), q in {2, 3} per state, "
                     "sum_i 4^N_i x 2 Pauli strings x q per step",
                     {"nstates": len(ns), "sum_4n": float(sum(4.0 ** n for n in ns)), "precision": precision,
                      "parallelism": f"state-list split x{world}"})
    line["e2e"] = {"value": units_all * args.steps / (e2e_ms * 1e-3), "unit": "Pauli-strings*q/s",
                   "h2d_bytes_per_step": int(sum(16 * (1 << n) for n in ns)),
                   "d2h_bytes_per_step": int(8 * len(ns) * (len(qs) + 1))}
    if precision == "fp32":
        o32 = sum(fp32_path_ops(n, len(qs))[0] * float(1 << n) for n in my_ns)
        o64 = sum(fp32_path_ops(n, len(qs))[1] * float(1 << n) for n in my_ns)
        line["roofline"] = roofline_fp32(o32, o64, total_ms / args.steps, gpu.ctx.probe_fp32_peak(),
                                         gpu.ctx.probe_fp64_peak())
        line["roofline"]["work"] += ", summed over the states"
    else:
        ops = sum(fp64_ops_per_x(n, len(qs)) * float(1 << n) for n in my_ns)
        line["roofline"] = roofline_fp64(ops, total_ms / args.steps, gpu.ctx.probe_fp64_peak(),
                                         "(n + 8) 2^n FP64 ops per X-string (q = 2 and 3), summed over the states")
    line["gpu_launches"] = int(launches)
    line["clocks"] = clocks
    if world == 1:
        # the repo's own per-state calls, and the plain GPU form (one state per call) on a
        # seeded subset of 64 states scaled by 4^N
        t0 = time.perf_counter()
        per_state_ms = 0.0
        for p in psis:
            _, ms = gpu.timed(lambda p=p: gpu.ctx.sre(p, qs, prec))
            per_state_ms += ms
        sub = np.random.default_rng(64).choice(len(ns), size=64, replace=False)
        plain_ms = 0.0
        for i in sub:
            _, ms = gpu.timed(lambda i=i: gpu.ctx.sre(psis[i], qs, hm.HM_PLAIN))
            plain_ms += ms
        scale = sum(4.0 ** n for n in ns) / sum(4.0 ** ns[i] for i in sub)
        vals, _ = gpu.ctx.sre_batched(psis, qs, prec)
        line["compare"] = {
            "per_state_hm_sre_ms": per_state_ms,
            "batched_e2e_ms": e2e_ms / args.steps,
            "speedup_vs_per_state_calls": per_state_ms / (e2e_ms / args.steps),
            "plain_ms_estimate": plain_ms * scale,
            "plain_sample": "64 seeded states, one HM_PLAIN call each, scaled by sum 4^N",
            "speedup_vs_plain": plain_ms * scale / (e2e_ms / args.steps),
            "wall_s": time.perf_counter() - t0,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_batched_sample(ns, psis, qs, 15.0)
        line["config"]["values_head"] = [float(v) for v in vals[:4, 0]]
    return line


def bench_grad(args, cfg, gpu, world, rank, dist):
    n = cfg["n"]
    psi = make_state(1 << n, cfg["seed"])
    hm = gpu.hm

    def step():
        _, ms = gpu.timed(lambda: gpu.ctx.sre_grad(psi, 2.0))
        return gpu.ctx.last_kernel_ms(), gpu.ctx.last_launch_count()

    total_ms, launches, clocks = run_steps(args, gpu, step, world, dist)
    units = 4.0 ** n
    value = units * args.steps / (total_ms * 1e-3)

    def e2e_step():
        _, ms = gpu.timed(lambda: gpu.ctx.sre_grad(psi, 2.0))
        return ms, 0

    e2e_ms, _, _ = run_steps(argparse.Namespace(warmup=1, steps=args.steps), gpu, e2e_step, world, dist)
    fwd = []
    for _ in range(args.steps + 1):
        gpu.timed(lambda: gpu.ctx.sre(psi, (2.0,), hm.HM_FP64))
        fwd.append(gpu.ctx.last_kernel_ms())
    fwd_ms = float(np.median(fwd[1:]))
    adj_ms = total_ms / args.steps
    line = base_line(args, args.config, f"Pauli-strings/s for the adjoint dSRE_2/dpsi N={n}", "Pauli-strings/s",
                     value, world, total_ms, "f64",
                     f"value and gradient of SRE_2 w.r.t. Re psi and Im psi, N={n}: 4^{n} Pauli strings per step",
                     {"n": n, "seed": cfg["seed"], "parallelism": "replicas only",
                      "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms})
    line["roofline"] = roofline_fp64(2 * fp64_ops_per_x(n) * float(1 << n), adj_ms, gpu.ctx.probe_fp64_peak(),
                                     "2 (n + 6) 2^n FP64 ops per X-string (forward and backward transform)")
    line["e2e"] = {"value": units * args.steps / (e2e_ms * 1e-3), "unit": "Pauli-strings/s",
                   "h2d_bytes_per_step": int(16 * (1 << n)), "d2h_bytes_per_step": int(16 * (1 << n) + 8)}
    line["gpu_launches"] = int(launches)
    line["clocks"] = clocks
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_grad(n, cfg["seed"])
    return line


def bench_mana(args, cfg, gpu, world, rank, dist):
    hm = gpu.hm
    L = cfg["L"]
    psi = make_state(3 ** L, cfg["seed"])
    if cfg["kind"] == "mana_pure":
        call = lambda: gpu.ctx.mana_pure(psi)  # noqa: E731
        units = 9.0 ** L
        name = f"phase-points/s for pure-state Mana, {L} qutrits"
        work = f"Mana of a {L}-qutrit pure state: 3^{L} ternary X-strings x 3^{L}-point transforms = 9^{L} phase points"
        h2d = 16 * 3 ** L
        extra = {"L": L}
    else:
        rho = hm.reduced_density_matrix(hm.StateVec(psi, q=3), cfg["keep"], side="right").data
        call = lambda: gpu.ctx.mana_mixed(rho)  # noqa: E731
        N = cfg["keep"]
        units = 9.0 ** N
        name = f"phase-points/s for mixed-state Mana, {3 ** N}x{3 ** N} density matrix"
        work = (f"Mana of the {3 ** N}x{3 ** N} reduced density matrix of a {L}-qutrit state (4 qutrits traced "
                f"out): 9^{N} phase points")
        h2d = 16 * 9 ** N
        extra = {"L": L, "N": N}
    res = {}

    def step():
        def c():
            res["v"] = call()
        gpu.timed(c)
        return gpu.ctx.last_kernel_ms(), gpu.ctx.last_launch_count()

    total_ms, launches, clocks = run_steps(args, gpu, step, world, dist)
    value = units * args.steps / (total_ms * 1e-3)

    def e2e_step():
        _, ms = gpu.timed(call)
        return ms, 0

    e2e_ms, _, _ = run_steps(argparse.Namespace(warmup=1, steps=args.steps), gpu, e2e_step, world, dist)
    extra["mana"] = float(res["v"])
    line = base_line(args, args.config, name, "phase-points/s", value, world, total_ms, "f64", work, extra)
    if cfg["kind"] == "mana_pure":
        # per X-string: L 3^(L-1) radix-3 butterflies (12 FP64 ops: 6 add/sub + 6 FMA),
        # 3^L gather-multiplies (6 ops) and 3^L moduli (4 ops + sqrt)
        ops = (L * 3 ** (L - 1) * 12 + 3 ** L * 10) * float(3 ** L)
        line["roofline"] = roofline_fp64(ops, total_ms / args.steps, gpu.ctx.probe_fp64_peak(),
                                         "(12 L 3^(L-1) + 10 3^L) FP64 ops per ternary X-string")
    else:
        N = cfg["keep"]
        # per leg every one of the 9^N outputs is a 9-term complex sum
        ops = N * 9 ** N * 9 * 8.0
        line["roofline"] = roofline_fp64(ops, total_ms / args.steps, gpu.ctx.probe_fp64_peak(),
                                         "N 9^N 9 complex multiply-adds (8 FP64 ops each)")
    line["e2e"] = {"value": units * args.steps / (e2e_ms * 1e-3), "unit": "phase-points/s",
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 8}
    line["gpu_launches"] = int(launches)
    line["clocks"] = clocks
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = (cpu_mana_pure(L, cfg["seed"], 10.0) if cfg["kind"] == "mana_pure"
                                else cpu_mana_mixed(rho))
    return line


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    cfg = CONFIGS[args.config]
    gpu = Gpu(local)
    gpu.hm._native.set_param(gpu.hm._native.HM_PARAM_ENGINE, {"auto": 0, "stage": 1, "queue": 2}[args.engine])
    kind = cfg["kind"]
    if kind == "sre":
        line = bench_sre(args, cfg, gpu, world, rank, dist)
    elif kind == "mc":
        line = bench_mc(args, cfg, gpu, world, rank, dist)
    elif kind == "batched":
        line = bench_batched(args, cfg, gpu, world, rank, dist)
    elif kind == "grad":
        line = bench_grad(args, cfg, gpu, world, rank, dist)
    else:
        line = bench_mana(args, cfg, gpu, world, rank, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    gpu.ctx.close()
    return 0


def run_reference(args):
    """The oracle (C restatement of the reference's :threads backend) on the host cores,
    on the configuration's workload; rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    cfg = CONFIGS[args.config]
    kind = cfg["kind"]
    vals, base = [], None
    for i in range(args.warmup + args.steps):
        secs = max(2.0, 90.0 / (args.warmup + args.steps))
        if kind == "sre":
            base = cpu_sre_sample(cfg["n"], cfg["seed"], cfg["qs"], secs)
            metric = f"Pauli-strings/s for exact SRE q={','.join(f'{q:g}' for q in cfg['qs'])} N={cfg['n']}"
            units = 4.0 ** cfg["n"]
        elif kind == "mc":
            base = cpu_mc_sample(cfg["n"], cfg["seed"], cfg["nbeta"], 10, cfg["stream_seed"])
            metric = f"Pauli-strings/s for MC_SRE q=2 N={cfg['n']} ({cfg['nbeta'] * cfg['nsamples']} proposals)"
            units = cfg["nbeta"] * cfg["nsamples"] * float(1 << cfg["n"])
        elif kind == "batched":
            ns, psis = batched_states(cfg)
            base = cpu_batched_sample(ns, psis, cfg["qs"], secs)
            metric = "Pauli-strings*q/s for batched exact SRE (512 states, N 8..18, q 2,3)"
            units = sum(4.0 ** n for n in ns) * len(cfg["qs"])
        elif kind == "grad":
            base = cpu_grad(cfg["n"], cfg["seed"])
            metric = f"Pauli-strings/s for the adjoint dSRE_2/dpsi N={cfg['n']}"
            units = 4.0 ** cfg["n"]
        elif kind == "mana_pure":
            base = cpu_mana_pure(cfg["L"], cfg["seed"], secs)
            metric = f"phase-points/s for pure-state Mana, {cfg['L']} qutrits"
            units = 9.0 ** cfg["L"]
        else:
            import hadamag_b200 as hm
            psi = make_state(3 ** cfg["L"], cfg["seed"])
            rho = hm.StateVec(psi, q=3)
            from oracle import oracle as O
            r = O.reduced_density_matrix(psi, 3, cfg["keep"], side="right")
            del rho
            base = cpu_mana_mixed(r)
            metric = f"phase-points/s for mixed-state Mana, {3 ** cfg['keep']}x{3 ** cfg['keep']} density matrix"
            units = 9.0 ** cfg["keep"]
        if i >= args.warmup:
            vals.append(base["value"])
    value = float(np.mean(vals))
    line = {
        "metric": metric, "impl": "reference", "value": value, "unit": base["unit"], "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": units / value * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded complex-Gaussian states (numpy default_rng), normalised",
        "config": {"name": args.config, "sample": base["sample"], "extrapolated": True},
        "cpu_baseline": dict(base, value=value),
        "e2e": {"value": value, "unit": base["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "HadaMAG.jl is Julia and no Julia toolchain is installed; the timed CPU implementation is the "
                "C restatement of its :threads path (oracle/hm_oracle.c) on all host threads, each step a "
                "bounded sample of the workload extrapolated at the measured rate",
    }
    print(json.dumps(line), flush=True)
    return 0


def profile_case(args):
    """Short workload for ncu: hm_sre_range on Gray indices [k0, k0 + count) of the
    seeded n-qubit state, or the adjoint on the whole state (--grad), or pure-state Mana
    of a seeded L-qutrit state (--mana L).  Prints the sums and the device time."""
    import hadamag_b200 as hm
    hm._native.set_param(hm._native.HM_PARAM_ADJ_BATCH, args.adj_batch)
    hm._native.set_param(hm._native.HM_PARAM_ENGINE, {"auto": 0, "stage": 1, "queue": 2}[args.engine])
    ctx = hm._native.default_context(0)
    if args.mana:
        v = make_state(3 ** args.mana, args.mana)
        for _ in range(args.repeat):
            m = ctx.mana_pure(v)
        print(f"L={args.mana} mana={m:.15g} kernel_ms={ctx.last_kernel_ms():.3f}")
        return 0
    psi = make_state(1 << args.n, args.n)
    if args.grad:
        for _ in range(args.repeat):
            v, g = ctx.sre_grad(psi, args.q[0])
        print(f"n={args.n} grad: sre={v:.15g} |g|={np.linalg.norm(g):.6g} kernel_ms={ctx.last_kernel_ms():.3f}")
        return 0
    prec = hm.PRECISIONS[args.precision or "fp64"]
    for _ in range(args.repeat):
        p2, m = ctx.sre_range(psi, args.k0, args.k0 + args.count, tuple(args.q), prec)
    print(f"n={args.n} k=[{args.k0},{args.k0 + args.count}) p2={p2.sum():.17g} m={m.sum(axis=1)} "
          f"kernel_ms={ctx.last_kernel_ms():.3f} launches={ctx.last_launch_count()}")
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 3 for the N = 20 and batched configurations; enough "
                         "steps for about a second of timed work for the short ones)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"],
                    help="override the configuration's precision (exact-SRE and batched configurations)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--engine", default="auto", choices=["auto", "stage", "queue"],
                    help="two-pass sweep of the single-state entry points: automatic (the tuned choice, else "
                         "the stage kernels), the stage kernels or the persistent queue")
    ap.add_argument("--profile-case", action="store_true", help="run the short ncu workload instead")
    ap.add_argument("--n", type=int, default=20)
    ap.add_argument("--k0", type=int, default=1024)
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--q", type=float, nargs="+", default=[2.0])
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--grad", action="store_true")
    ap.add_argument("--adj-batch", type=int, default=0)
    ap.add_argument("--mana", type=int, default=0)
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.steps is None:
        args.steps = DEFAULT_STEPS.get(args.config, 3) if args.impl == "ours" else 3
    if args.steps < 1:
        ap.error("--steps must be >= 1")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
