"""Generate the large adjoint and Mana fixtures from the oracle (test infrastructure).

    python tests/golden/gen_large.py [--threads T] [--only grad|mana]

grad_n18_seed18.json: the oracle's SRE_2 gradient (oracle/hm_oracle.c or_sre_grad) of
the seeded 18-qubit state of the adjoint configuration (numpy default_rng(18), real
then imaginary parts N(0, 1), normalised): the value, 64 seeded coordinates, the largest
modulus and 4 seeded projections sum_r w_r0 Re g_r + w_r1 Im g_r with w from
default_rng(1000 + k).normal(size=(2^18, 2)).

mana_pure_L10_L11.json: the oracle's pure-state Mana (or_mana_sum over every ternary
X-string, src/Mana.jl:19-92) of the seeded 10- and 11-qutrit states (default_rng(L)).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def state(dim, seed):
    g = np.random.default_rng(seed)
    v = g.normal(size=dim) + 1j * g.normal(size=dim)
    return v / np.linalg.norm(v)


def gen_grad(threads):
    n = 18
    psi = state(1 << n, 18)
    t0 = time.time()
    v, g = O.sre_grad(psi, 2, nthreads=threads)
    idx = np.random.default_rng(6418).integers(0, 1 << n, size=64)
    proj = []
    for k in range(4):
        w = np.random.default_rng(1000 + k).normal(size=(1 << n, 2))
        proj.append(float(np.sum(w[:, 0] * g.real + w[:, 1] * g.imag)))
    out = {"n": n, "seed": 18, "q": 2, "sre": v, "idx": [int(i) for i in idx],
           "g_re": [float(g[i].real) for i in idx], "g_im": [float(g[i].imag) for i in idx],
           "max_abs": float(np.max(np.abs(g))), "proj": proj,
           "generator": "tests/golden/gen_large.py (oracle or_sre_grad)", "seconds": round(time.time() - t0, 1)}
    with open(os.path.join(HERE, "grad_n18_seed18.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("grad", out["sre"], out["seconds"])


def gen_mana(threads):
    out = {}
    for L in (10, 11):
        psi = state(3 ** L, L)
        t0 = time.time()
        s = O.mana_sum(psi, 1, 3 ** L, nthreads=threads)
        out[str(L)] = {"L": L, "seed": L, "sum": s, "mana": float(np.log2(s) / np.log2(3.0)),
                       "seconds": round(time.time() - t0, 1)}
        print("mana", L, out[str(L)])
    out["generator"] = "tests/golden/gen_large.py (oracle or_mana_sum)"
    with open(os.path.join(HERE, "mana_pure_L10_L11.json"), "w") as f:
        json.dump(out, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", choices=["grad", "mana"], default=None)
    args = ap.parse_args()
    O.build()
    if args.only in (None, "grad"):
        gen_grad(args.threads)
    if args.only in (None, "mana"):
        gen_mana(args.threads)


if __name__ == "__main__":
    main()
