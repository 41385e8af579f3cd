"""Generate the N = 20 exact-SRE fixture from the oracle (test infrastructure).

    python tests/golden/gen_n20.py [--threads T]

The state is the seeded normalised complex Gaussian of the N = 20 configuration
(numpy default_rng(20): real then imaginary parts N(0, 1), divided by the 2-norm), the
same vector bench.py times.  The oracle's fast path (oracle/hm_oracle.c,
or_sre_sums_fast: the Gray walk, build, FWHT and moments of src/SRE.jl:338-540 with
double-double sums) runs over all 2^20 X-strings for q = 2 and q = 3 in one sweep, and
over four Gray sub-ranges that the GPU tests also run.  Writes tests/golden/n20_seed20.json
with the double-double sums and the finished (SRE, lost_norm) values.  Takes about 20
minutes on 8 cores.
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

N = 20
SEED = 20
QS = (2.0, 3.0)
# Gray sub-ranges [kb, ke) (0-based) checked one by one
SUBRANGES = [(1, 1025), (1024, 2048), ((1 << 19) - 100, (1 << 19) + 100), ((1 << 20) - 512, 1 << 20)]


def state():
    g = np.random.default_rng(SEED)
    v = g.normal(size=1 << N) + 1j * g.normal(size=1 << N)
    return v / np.linalg.norm(v)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    O.build()
    psi = state()
    t0 = time.time()
    sub = []
    for kb, ke in SUBRANGES:
        p2, m = O.sre_sums_fast(psi, QS, kb + 1, ke, nthreads=args.threads)
        sub.append({"k_begin": kb, "k_end": ke, "p2": p2.tolist(), "m": m.tolist()})
    p2, m = O.sre_sums_fast(psi, QS, 1, 1 << N, nthreads=args.threads)
    dim = float(1 << N)
    out = {
        "n": N, "seed": SEED, "qs": list(QS),
        "state": "numpy default_rng(20): normal(2^20) + 1j normal(2^20), normalised",
        "p2_dd": p2.tolist(), "m_dd": m.tolist(),
        "sre": [float(-np.log2((m[i, 0] + m[i, 1]) / dim)) for i in range(len(QS))],
        "lost_norm": float(abs(1.0 - (p2[0] + p2[1]) / dim)),
        "subranges": sub,
        "generator": "tests/golden/gen_n20.py (oracle or_sre_sums_fast)",
        "seconds": round(time.time() - t0, 1),
    }
    with open(os.path.join(HERE, "n20_seed20.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: out[k] for k in ("sre", "lost_norm", "seconds")}))


if __name__ == "__main__":
    main()
