"""Small exact-SRE workload for kernel profiling (ncu) and quick timing.

Runs hm_sre_range on a slice of Gray indices of a seeded N-qubit state, so that one
profiled launch of the two-pass stage kernel sees the full-size transform (2^(N-1)
points per X-string) while the whole run stays short:

    python hadamag.jl_b200/prof_case.py --n 20 --k0 1024 --count 256 --precision fp64

Prints the sums and the device time of the call.  With --grad it runs the adjoint
(hm_sre_grad, q = 2) on the whole n-qubit state instead; with --mana L, the pure-state
Mana of a seeded L-qutrit state.
"""
import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import hadamag_b200 as hm  # noqa: E402


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=20)
    ap.add_argument("--k0", type=int, default=1024, help="first Gray index")
    ap.add_argument("--count", type=int, default=256, help="number of X-strings")
    ap.add_argument("--precision", default="fp64", choices=sorted(hm.PRECISIONS))
    ap.add_argument("--q", type=float, nargs="+", default=[2.0])
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--grad", action="store_true", help="run the adjoint on the whole state")
    ap.add_argument("--adj-batch", type=int, default=0, help="X-strings per adjoint stage (0: default)")
    ap.add_argument("--mana", type=int, default=0, help="run Mana on a seeded L-qutrit state instead")
    args = ap.parse_args()
    hm._native.set_param(hm._native.HM_PARAM_ADJ_BATCH, args.adj_batch)
    if args.mana:
        g = np.random.default_rng(args.mana)
        v = g.normal(size=3 ** args.mana) + 1j * g.normal(size=3 ** args.mana)
        v /= np.linalg.norm(v)
        ctx = hm._native.default_context(0)
        for _ in range(args.repeat):
            m = ctx.mana_pure(v)
        print(f"L={args.mana} mana={m:.15g} kernel_ms={ctx.last_kernel_ms():.3f}")
        return
    g = np.random.default_rng(args.n)
    psi = g.normal(size=1 << args.n) + 1j * g.normal(size=1 << args.n)
    psi /= np.linalg.norm(psi)
    ctx = hm._native.default_context(0)
    if args.grad:
        for _ in range(args.repeat):
            v, g = ctx.sre_grad(psi, args.q[0])
        print(f"n={args.n} grad: sre={v:.15g} |g|={np.linalg.norm(g):.6g} kernel_ms={ctx.last_kernel_ms():.3f}")
        return
    for _ in range(args.repeat):
        p2, m = ctx.sre_range(psi, args.k0, args.k0 + args.count, tuple(args.q), hm.PRECISIONS[args.precision])
    print(f"n={args.n} k=[{args.k0},{args.k0 + args.count}) p2={p2.sum():.17g} m={m.sum(axis=1)} "
          f"kernel_ms={ctx.last_kernel_ms():.3f} launches={ctx.last_launch_count()}")


if __name__ == "__main__":
    main()
