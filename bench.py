"""Benchmark: exact stabilizer Renyi entropy, q = 2, N = 20 qubits, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--precision fp64|fp32]
    torchrun --nnodes=1 --nproc-per-node N --master-addr 127.0.0.1 bench.py --gpus N

One step is one full exact SRE of a 20-qubit state: all 2^20 Pauli X-strings, each a
2^20-point Walsh-Hadamard transform, i.e. 4^20 Pauli strings.  The state is a seeded,
normalised complex-Gaussian vector (numpy default_rng(20)), synthetic: the reference
publishes no benchmark input.  With N GPUs the Gray-code range is split across ranks
(strong scaling: the job is fixed); the ranks exchange their double-double partial sums
with one NCCL all_gather per step.

Printed (rank 0, one JSON line): `value` = Pauli strings per second of the whole job
with the state resident in HBM (device time, CUDA events, max over ranks); `e2e` = the
same metric through the C ABI call with a host-memory state, host-to-device copy and
result read-back inside the timed region; `roofline` = FP64-pipe operations of the
dominant kernel against the measured DADD rate of this GPU; `cpu_baseline` = the oracle
(a C restatement of the reference's :threads backend) on a bounded sample with all host
threads.  `--impl reference` times that CPU restatement alone on the same workload (the
reference itself is Julia, which this image does not ship).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 20
Q = 2.0
SEED = 20


def make_state(n, seed):
    g = np.random.default_rng(seed)
    v = g.normal(size=1 << n) + 1j * g.normal(size=1 << n)
    return v / np.linalg.norm(v)


def fp64_ops_per_x(n):
    """FP64-pipe operations of one X-string (n + 6) 2^n: n 2^n butterfly adds, 2 2^n
    for the product f = conj(psi(r)) psi(r ^ x), 4 2^n for the q = 2 moments."""
    return (n + 6) * (1 << n)


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


def cpu_baseline(n, seconds=12.0):
    """The oracle (C restatement of src/Backends/Threads.jl:108-159, OpenMP static
    partition) on a sample of Gray indices; returns Pauli strings / s."""
    from oracle import oracle as O
    O.build()
    psi = make_state(n, SEED)
    threads = os.cpu_count() or 1
    k0 = 1 << (n - 1)
    O.sre_sums(psi, 2, k0 + 1, k0 + threads, nthreads=threads)  # thread start-up and first touch
    t = time.perf_counter()
    O.sre_sums(psi, 2, k0 + 1, k0 + 2 * threads, nthreads=threads)
    dt = max(time.perf_counter() - t, 1e-3)
    count = max(threads, int(seconds / dt * 2 * threads) // threads * threads)
    t = time.perf_counter()
    O.sre_sums(psi, 2, k0 + 1, k0 + count, nthreads=threads)
    dt = time.perf_counter() - t
    return {"value": count * float(1 << n) / dt, "unit": "Pauli-strings/s", "cores": threads, "kind": "port",
            "sample": f"{count} X-strings (Gray indices {k0}..{k0 + count - 1}) of the N={n} state, "
                      f"{dt:.1f} s, oracle/hm_oracle.c compiled -O3 x86-64-v3 with OpenMP"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = N_QUBITS
    steps = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(n, seconds=max(2.0, 90.0 / (args.warmup + args.steps)))
        if i >= args.warmup:
            steps.append(r["value"])
        base = r
    value = float(np.mean(steps))
    line = {
        "metric": "Pauli-strings/s for exact SRE q=2 N=20", "impl": "reference", "value": value,
        "unit": "Pauli-strings/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 4.0 ** n / value * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded complex-Gaussian 20-qubit state (numpy default_rng(20))",
        "config": {"workload": "exact SRE q=2, N=20 qubits (4^20 Pauli strings per step)", "n": n, "q": 2,
                   "sample": base["sample"]},
        "cpu_baseline": {"value": value, "unit": "Pauli-strings/s", "cores": base["cores"], "kind": "port",
                         "sample": base["sample"]},
        "e2e": {"value": value, "unit": "Pauli-strings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "HadaMAG.jl is Julia and no Julia toolchain is installed; the timed CPU implementation is the "
                "C restatement of its :threads exact-SRE path (oracle/hm_oracle.c) on all host threads",
    }
    print(json.dumps(line), flush=True)
    return 0


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
    import hadamag_b200 as hm
    from hadamag_b200 import shard

    n = N_QUBITS
    prec = hm.PRECISIONS[args.precision]
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = hm._native.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    psi_host = make_state(n, SEED)
    psi_dev = torch.from_numpy(psi_host.view(np.float64).copy()).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # larger than the 126 MB L2
    kb, ke = shard.gray_slice(n, rank, world)
    peak = ctx.probe_fp64_peak()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def step_device():
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        p2, m = ctx.sre_range_dev(psi_dev.data_ptr(), n, kb, ke, (Q,), prec)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), np.concatenate([p2, m.reshape(-1)]), ctx.last_launch_count()

    def step_e2e():
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        p2, m = ctx.sre_range(psi_host, kb, ke, (Q,), prec)  # host state: H2D inside the call
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), np.concatenate([p2, m.reshape(-1)])

    for _ in range(args.warmup):
        step_device()
    barrier()
    times, launches, partial = [], 0, None
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            ms, partial, nl = step_device()
            times.append(ms)
            launches += nl
        barrier()
    total_ms = float(np.sum(times))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        gathered = shard.allgather_partials(partial, device=dev)
    else:
        gathered = partial[None, :]
    sre, lost = shard.combine_partials(gathered, n, 1)
    pauli_per_step = 4.0 ** n
    value = pauli_per_step * args.steps / (total_ms * 1e-3)

    # end to end through the C ABI with the state in host memory
    for _ in range(1):
        step_e2e()
    barrier()
    e2e_times = []
    for _ in range(args.steps):
        ms, _ = step_e2e()
        e2e_times.append(ms)
    barrier()
    e2e_ms = float(np.sum(e2e_times))
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = pauli_per_step * args.steps / (e2e_ms * 1e-3)

    # roofline of the dominant kernel (the two-pass stage kernels run back to back inside
    # CUDA graphs; their average launch time is this rank's device time per step divided
    # by the stage launches, over the X-strings one launch covers)
    my_ms = float(np.sum(times)) / args.steps
    ops_per_step = fp64_ops_per_x(n) * float(ke - kb)
    achieved = ops_per_step / (my_ms * 1e-3)
    roofline = {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Top/s (FP64 pipe)",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "measured live on this GPU: register-resident DADD kernel (hm_probe_fp64_peak)",
                "algorithmic_ops_per_x": fp64_ops_per_x(n)}
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(prof) and args.precision in json.load(open(prof)):
        d = json.load(open(prof))[args.precision]
        roofline["traffic"] = d["dram_bytes_per_x"] * float(ke - kb)
        roofline["traffic_unit"] = "DRAM bytes (read + write) per step of this rank"
        roofline["traffic_note"] = d["note"]

    line = {
        "metric": "Pauli-strings/s for exact SRE q=2 N=20", "value": value, "unit": "Pauli-strings/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-butterflies/f64-reduction",
        "data": "synthetic: seeded complex-Gaussian 20-qubit state (numpy default_rng(20)), normalised",
        "config": {"workload": "exact SRE q=2, N=20 qubits: 2^20 X-strings x 2^20-point WHT = 4^20 Pauli strings "
                               "per step", "n": n, "q": 2, "precision": args.precision,
                   "parallelism": f"gray-range split x{world}", "l2": "flushed before every step (256 MiB write)",
                   "sre": float(sre[0]), "lost_norm": float(lost)},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "Pauli-strings/s", "h2d_bytes_per_step": int(world * 16 * (1 << n)),
                "d2h_bytes_per_step": int(world * 8 * 4)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(n)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
