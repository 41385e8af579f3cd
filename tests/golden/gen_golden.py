"""Generate tests/golden/golden.json: small fixtures that pin the C oracle.

HadaMAG.jl holds no golden SRE / Mana values (its tests compare backends on unseeded
random states, test/SRE_test.jl:48-55, test/Mana_test.jl:1-12) and Julia is not
available here, so these fixtures come from a second, independent restatement of the
reference's definitions in plain Python/numpy, written for small sizes only:

  * Gray tables: src/Basis.jl:14-27 (generate_binary), 76-106 (generate_binary_
    splitted), 123-164 (integer_to_gray, generate_general), src/Helpers.jl:18-23
    (partition_counts);
  * exact SRE by the naive O(8^n) definition, src/SRE.jl:643-749 (expval_pauli_mask,
    naive_SRE), including the reference's value -log2(sum (e^2)^q / 2^n) for q != 2;
  * analytic known answers: products of T states, GHZ (stabilizer) states;
  * pure-state Mana, src/Mana.jl:19-113 with src/Helpers.jl:249-292, and mixed-state
    Mana, src/Mana.jl:123-314;
  * one Metropolis chain with an explicit proposal stream, src/SRE.jl:110-192.

Run:  python tests/golden/gen_golden.py   (writes golden.json next to this file)
"""
import itertools
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# ----------------------------------------------------------------------------- Gray codes
def gray_binary(n):
    N = 1 << n
    codes = [k ^ (k >> 1) for k in range(N)]
    flips = [((codes[k] ^ codes[k + 1]) & -(codes[k] ^ codes[k + 1])).bit_length() for k in range(N - 1)]
    return codes, flips


def partition_counts(n, P):
    base, rem = divmod(n, P)
    counts = [base + 1 if i < rem else base for i in range(P)]
    displs = [sum(counts[:i]) for i in range(P)]
    return counts, displs


def integer_to_gray(val, q, n):
    digits = []
    for _ in range(n):
        digits.append(val % q)
        val //= q
    shift, gray = 0, [0] * n
    for i in range(n - 1, -1, -1):
        gray[i] = (digits[i] + shift) % q
        shift += q - gray[i]
    return gray


def gray_general(n, q):
    N = q ** n
    cols = [integer_to_gray(k, q, n) for k in range(N)]
    flips = []
    for k in range(N - 1):
        flips.append(next(i + 1 for i in range(n) if cols[k][i] != cols[k + 1][i]))
    return cols, flips


# ----------------------------------------------------------------------------- SRE
def expval(psi, x, z):
    n = int(np.log2(psi.size))
    b = np.arange(psi.size)
    sign = np.where(np.array([bin(int(v) & z).count("1") & 1 for v in b]), -1.0, 1.0)
    s = np.sum(np.conj(psi[b ^ x]) * psi * sign)
    ph = [1, 1j, -1, -1j][bin(x & z).count("1") & 3]
    return float(np.real(ph * s))


def naive_sre(psi, q):
    n = int(np.log2(psi.size))
    tot = 0.0
    for idx in range(4 ** n):
        x = z = 0
        t = idx
        for j in range(n):
            d = t & 3
            if d in (1, 2):
                x |= 1 << j
            if d in (2, 3):
                z |= 1 << j
            t >>= 2
        e = expval(psi, x, z)
        tot += (e * e) ** q
    return -np.log2(tot / psi.size)


def t_state(n):
    t = np.array([1, np.exp(1j * np.pi / 4)]) / np.sqrt(2)
    v = np.array([1.0 + 0j])
    for _ in range(n):
        v = np.kron(v, t)
    return v


def ghz(n):
    v = np.zeros(1 << n, dtype=complex)
    v[0] = v[-1] = 1 / np.sqrt(2)
    return v


def rand_state(dim, seed):
    g = np.random.default_rng(seed)
    v = g.normal(size=dim) + 1j * g.normal(size=dim)
    return v / np.linalg.norm(v)


# ----------------------------------------------------------------------------- Mana
def h3(v, L):
    w = np.exp(2j * np.pi / 3)
    D = np.array([[1, 1, 1], [1, w, w * w], [1, w * w, w]])
    a = v.reshape([3] * L)  # axis 0 = most significant digit
    for ax in range(L):
        a = np.moveaxis(np.tensordot(D, a, axes=([1], [ax])), 0, ax)
    return a.reshape(-1)


def tern_digits(r, L):
    return [(r // 3 ** s) % 3 for s in range(L)]


def tern_num(d):
    return sum(v * 3 ** s for s, v in enumerate(d))


def mana_pure(psi):
    L = int(round(np.log(psi.size) / np.log(3)))
    D = psi.size
    S = 0.0
    for x in range(D):
        xd = tern_digits(x, L)
        inv = np.empty(D, dtype=complex)
        for r in range(D):
            rd = tern_digits(r, L)
            a = psi[tern_num([(rd[s] + xd[s]) % 3 for s in range(L)])]
            b = psi[tern_num([((3 - rd[s]) % 3 + xd[s]) % 3 for s in range(L)])]
            inv[r] = np.conj(a) * (b / D)
        S += np.sum(np.abs(h3(inv, L)))
    return np.log2(S) / np.log2(3)


def phase_point_M():
    w = np.exp(2j * np.pi / 3)
    X = np.zeros((3, 3), complex)
    for k in range(3):
        X[(k + 1) % 3, k] = 1
    Z = np.diag([w ** k for k in range(3)])
    T = {}
    for a in range(3):
        for ap in range(3):
            T[3 * a + ap] = w ** ((-2 * a * ap) % 3) * (np.linalg.matrix_power(Z, a) @ np.linalg.matrix_power(X, ap))
    A0 = sum(T.values()) / 3
    M = np.zeros((9, 9), complex)
    for u in range(9):
        Au = T[u] @ A0 @ T[u].conj().T
        M[u, :] = Au.T.reshape(-1, order="F")
    return M


def mana_mixed(rho):
    dim = rho.shape[0]
    N = int(round(np.log(dim) / np.log(3)))
    op = 9 ** N
    v = np.zeros(op, complex)
    for c0 in range(dim):
        jd = [(c0 // 3 ** (N - 1 - k)) % 3 for k in range(N)]
        for r0 in range(dim):
            idg = [(r0 // 3 ** (N - 1 - k)) % 3 for k in range(N)]
            p = 0
            for k in range(N):
                p = p * 9 + 3 * idg[k] + jd[k]
            v[p] = rho[r0, c0]
    M = phase_point_M()
    a = v.reshape([9] * N)  # axis 0 = leg 1 (most significant)
    for ax in range(N):
        a = np.moveaxis(np.tensordot(M, a, axes=([1], [ax])), 0, ax)
    return float(np.log2(np.sum(np.abs(a)) / dim))


# ----------------------------------------------------------------------------- MC chain
def fwht(v):
    v = v.copy()
    h = 1
    while h < v.size:
        for i in range(0, v.size, 2 * h):
            a = v[i:i + h].copy()
            b = v[i + h:i + 2 * h].copy()
            v[i:i + h] = a + b
            v[i + h:i + 2 * h] = a - b
        h *= 2
    return v


def mc_chain(psi, beta, prop_delta, rs):
    dim = psi.size
    X1, X2 = psi.real, psi.imag
    T1, T2 = X1 + X2, X2 - X1
    idx = np.arange(dim)

    def sample(mask):
        g = X1 * T1[idx ^ mask] + X2 * T2[idx ^ mask]
        F = fwht(g)
        return np.sum(F * F) / dim, np.sum((F * F) ** 2)

    p2_0, m0 = sample(0)
    cur, prob, m2, p2 = 0, 1e-120, 0.0, p2_0
    sM2 = sM2sq = sP2 = 0.0
    masks = []
    for t in range(len(rs)):
        prop = cur ^ int(prop_delta[t])
        p2p, mp = sample(prop)
        pb = mp ** beta
        if rs[t] < pb / prob and prop != 0:
            cur, prob, m2, p2 = prop, pb, -np.log2(mp), p2p
        sM2 += m2
        sM2sq += m2 * m2
        sP2 += p2
        masks.append(cur)
    n = len(rs)
    return [sM2 / n, sM2sq / n, m0 / dim, sP2 / n, n], masks


def main():
    out = {"gray_binary": {}, "gray_split": [], "gray_general": {}, "sre": [], "mana_pure": [], "mana_mixed": [],
           "mc_chain": []}
    for n in range(0, 6):
        c, f = gray_binary(n)
        out["gray_binary"][str(n)] = {"codes": c, "flips": f}
    for n, P in itertools.product(range(2, 7), range(1, 6)):
        counts, displs = partition_counts(1 << n, P)
        for rank in range(P):
            codes = [(displs[rank] + j) ^ ((displs[rank] + j) >> 1) for j in range(counts[rank])]
            flips = [((codes[j] ^ codes[j + 1]) & -(codes[j] ^ codes[j + 1])).bit_length()
                     for j in range(len(codes) - 1)]
            out["gray_split"].append({"n": n, "P": P, "rank": rank, "code_off": displs[rank], "codes": codes,
                                      "flips": flips})
    for n, q in [(2, 3), (1, 4), (3, 3), (2, 5), (4, 3)]:
        cols, flips = gray_general(n, q)
        out["gray_general"][f"{n},{q}"] = {"columns": cols, "flips": flips}

    for n in range(1, 5):
        for q in (2, 3):
            psi = rand_state(1 << n, 1000 + 10 * n + q)
            out["sre"].append({"kind": "random", "n": n, "q": q, "seed": 1000 + 10 * n + q,
                               "re": psi.real.tolist(), "im": psi.imag.tolist(), "sre": naive_sre(psi, q)})
    for n in range(1, 7):
        out["sre"].append({"kind": "t_state", "n": n, "q": 2, "sre": n * np.log2(4 / 3)})
        out["sre"].append({"kind": "t_state", "n": n, "q": 3, "sre": n * np.log2(8 / 5)})
        out["sre"].append({"kind": "ghz", "n": n, "q": 2, "sre": 0.0})
    for L in (1, 2):
        psi = rand_state(3 ** L, 2000 + L)
        out["mana_pure"].append({"L": L, "seed": 2000 + L, "re": psi.real.tolist(), "im": psi.imag.tolist(),
                                 "mana": mana_pure(psi)})
    for N in (1, 2):
        psi = rand_state(3 ** N, 3000 + N)
        rho = np.outer(psi, psi.conj())
        out["mana_mixed"].append({"N": N, "seed": 3000 + N, "re": psi.real.tolist(), "im": psi.imag.tolist(),
                                  "mana": mana_mixed(rho)})
    psi = rand_state(8, 4000)
    g = np.random.default_rng(4001)
    prop = [int(v) for v in g.integers(0, 8, size=24)]
    rs = g.random(24).tolist()
    for beta in (0.0, 0.5, 1.0):
        res, masks = mc_chain(psi, beta, prop, rs)
        out["mc_chain"].append({"n": 3, "beta": beta, "re": psi.real.tolist(), "im": psi.imag.tolist(),
                                "prop_delta": prop, "rs": rs, "out5": res, "masks": masks})
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
