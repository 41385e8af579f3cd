"""The C oracle against the golden fixtures (tests/golden/gen_golden.py restates the
reference's definitions independently) and against the Gray-code properties the
reference's own tests assert (test/Basis_test.jl:3-156)."""
import numpy as np
import pytest

from conftest import ghz, rand_state, t_state


def test_gray_binary_pins(oracle, golden):
    for n_str, g in golden["gray_binary"].items():
        n = int(n_str)
        codes, flips = oracle.gray_binary(n)
        assert codes.tolist() == g["codes"]
        assert flips.tolist() == g["flips"]


def test_gray_binary_reference_properties(oracle):
    # test/Basis_test.jl:4-22
    for n in range(0, 5):
        codes, flips = oracle.gray_binary(n)
        N = 1 << n
        assert len(codes) == N and len(flips) == max(0, N - 1)
        assert codes[0] == 0
        for k in range(N - 1):
            diff = int(codes[k]) ^ int(codes[k + 1])
            assert bin(diff).count("1") == 1
            assert flips[k] == (diff & -diff).bit_length()
            assert int(codes[k + 1]) == (k + 1) ^ ((k + 1) >> 1)


def test_gray_split_pins(oracle, golden):
    # test/Basis_test.jl:27-66: concatenated slices == full table, total flips = N - min(N, P)
    by = {}
    for g in golden["gray_split"]:
        codes, flips, off = oracle.gray_binary_split(g["n"], g["rank"], g["P"])
        assert off == g["code_off"]
        assert codes.tolist() == g["codes"]
        assert flips.tolist() == g["flips"]
        by.setdefault((g["n"], g["P"]), []).append((g["rank"], codes.tolist(), len(flips)))
    for (n, P), parts in by.items():
        parts.sort()
        full = sum((p[1] for p in parts), [])
        assert full == oracle.gray_binary(n)[0].tolist()
        N = 1 << n
        assert sum(p[2] for p in parts) == N - min(N, P)


def test_gray_general_pins(oracle, golden):
    # test/Basis_test.jl:70-88
    for key, g in golden["gray_general"].items():
        n, q = map(int, key.split(","))
        xt, flips = oracle.gray_general(n, q)
        assert xt.shape == (n, q ** n)
        assert xt.T.tolist() == g["columns"]
        assert flips.tolist() == g["flips"]
        # single-digit steps, each a +1 mod q on the flipped digit (asserted by
        # src/Mana.jl:81-82 for q = 3)
        for k in range(q ** n - 1):
            d = np.nonzero(xt[:, k] != xt[:, k + 1])[0]
            assert len(d) == 1 and d[0] + 1 == flips[k]
            assert (xt[d[0], k + 1] - xt[d[0], k]) % q == 1


def test_partition_counts(oracle):
    for n in range(0, 40):
        for P in range(1, 9):
            c, d = oracle.partition_counts(n, P)
            assert c.sum() == n and max(c) - min(c) <= 1 and list(c) == sorted(c, reverse=True)
            assert d[0] == 0 and all(d[i + 1] == d[i] + c[i] for i in range(P - 1))


def test_sre_golden(oracle, golden):
    for g in golden["sre"]:
        n, q = g["n"], g["q"]
        if g["kind"] == "random":
            psi = np.array(g["re"]) + 1j * np.array(g["im"])
        elif g["kind"] == "t_state":
            psi = t_state(n)
        else:
            psi = ghz(n)
        v, lost = oracle.sre(psi, q)
        assert v == pytest.approx(g["sre"], rel=1e-12, abs=1e-12)
        assert lost < 1e-13


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7])
@pytest.mark.parametrize("q", [2, 3])
def test_sre_fast_equals_naive(oracle, n, q):
    psi = rand_state(1 << n, 77 + n)
    assert oracle.sre(psi, q)[0] == pytest.approx(oracle.naive_sre(psi, q), rel=1e-12)


def test_sre_threads_equals_serial(oracle):
    # test/SRE_test.jl:217-224 compares :serial and :threads
    psi = rand_state(1 << 9, 9)
    assert oracle.sre(psi, 2, nthreads=1)[0] == pytest.approx(oracle.sre(psi, 2, nthreads=7)[0], rel=1e-14)


def test_sre_sums_additive_over_ranges(oracle):
    psi = rand_state(1 << 8, 8)
    full = oracle.sre_sums(psi, 2, 1, 256)
    a = oracle.sre_sums(psi, 2, 1, 100)
    b = oracle.sre_sums(psi, 2, 101, 256)
    assert a[0] + b[0] == pytest.approx(full[0], rel=1e-14)
    assert a[1] + b[1] == pytest.approx(full[1], rel=1e-14)
    # Parseval: sum over all Pauli strings of <P>^2 = 2^n for a normalised state
    assert full[0] == pytest.approx(256.0, rel=1e-13)


def test_mana_golden(oracle, golden):
    for g in golden["mana_pure"]:
        psi = np.array(g["re"]) + 1j * np.array(g["im"])
        assert oracle.mana_pure(psi) == pytest.approx(g["mana"], rel=1e-12)
    for g in golden["mana_mixed"]:
        psi = np.array(g["re"]) + 1j * np.array(g["im"])
        assert oracle.mana_mixed(np.outer(psi, psi.conj())) == pytest.approx(g["mana"], rel=1e-12, abs=1e-12)


def test_mana_known_answers(oracle):
    for L in (1, 2, 3):
        psi = np.zeros(3 ** L, complex)
        psi[0] = 1
        assert abs(oracle.mana_pure(psi)) < 1e-14
        assert abs(oracle.mana_mixed(np.eye(3 ** L) / 3 ** L)) < 1e-13
        psi = rand_state(3 ** L, 5 + L)
        # the two log bases (src/Backends/Threads.jl:270 vs src/Mana.jl:311)
        assert oracle.mana_mixed(np.outer(psi, psi.conj())) == pytest.approx(np.log2(3) * oracle.mana_pure(psi),
                                                                             rel=1e-12)


def test_mc_chain_golden(oracle, golden):
    for g in golden["mc_chain"]:
        psi = np.array(g["re"]) + 1j * np.array(g["im"])
        out5, masks = oracle.mc_sre_beta(psi, 2, g["beta"], np.array(g["prop_delta"], dtype=np.uint64),
                                         np.array(g["rs"]))
        assert np.allclose(out5, g["out5"], rtol=1e-12, atol=1e-14)
        assert masks.tolist() == g["masks"]


def test_simpson(oracle):
    x = np.linspace(0, 1, 13)
    assert oracle.simpson_uniform(x, x ** 3) == pytest.approx(0.25, rel=1e-14)
    assert np.isnan(oracle.simpson_uniform(np.linspace(0, 1, 4), np.ones(4)))


def test_grad_matches_finite_differences(oracle):
    n = 4
    psi = rand_state(1 << n, 44)
    v, g = oracle.sre_grad(psi, 2)
    h = 1e-6
    rng = np.random.default_rng(1)
    for _ in range(8):
        r = int(rng.integers(0, 1 << n))
        for comp in (1.0, 1j):
            p, m = psi.copy(), psi.copy()
            p[r] += h * comp
            m[r] -= h * comp
            fd = (oracle.sre(p, 2)[0] - oracle.sre(m, 2)[0]) / (2 * h)
            an = g[r].real if comp == 1.0 else g[r].imag
            assert an == pytest.approx(fd, rel=1e-5, abs=1e-8)


def _apply_2gate_numpy(psi, q, gate, s1, s2):
    """Independent restatement of apply_2gate! (src/State.jl:279-344) by tensor
    contraction: site s is axis n - s of the C-order reshaped state."""
    n = int(round(np.log(psi.size) / np.log(q)))
    t = psi.reshape((q,) * n)
    a1, a2 = n - s1, n - s2
    g = np.asarray(gate).reshape(q, q, q, q)  # [o1, o2, d1, d2]
    t = np.moveaxis(t, (a1, a2), (0, 1))
    t = np.einsum("abcd,cd...->ab...", g, t)
    return np.moveaxis(t, (0, 1), (a1, a2)).reshape(-1)


@pytest.mark.parametrize("q,n", [(2, 2), (2, 5), (3, 2), (3, 4)])
def test_oracle_apply_2gate(oracle, q, n):
    rng = np.random.default_rng(10 * q + n)
    psi = rand_state(q ** n, 3 + n)
    for s1 in range(1, n + 1):
        for s2 in range(1, n + 1):
            if s1 == s2:
                continue
            gate = rng.normal(size=(q * q, q * q)) + 1j * rng.normal(size=(q * q, q * q))
            out = oracle.apply_2gate(psi, q, gate, s1, s2)
            assert np.allclose(out, _apply_2gate_numpy(psi, q, gate, s1, s2), atol=1e-12)


def test_oracle_apply_2gate_known_answers(oracle):
    # CNOT with control site s1 and target s2 (row/column index b1 * 2 + b2)
    cnot = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)
    n = 4
    for i in range(1 << n):
        e = np.zeros(1 << n, complex)
        e[i] = 1
        out = oracle.apply_2gate(e, 2, cnot, 3, 1)  # control site 3 (bit 2), target site 1 (bit 0)
        j = i ^ 1 if (i >> 2) & 1 else i
        assert out[j] == 1 and np.count_nonzero(out) == 1


def test_oracle_brick_wall_is_gate_sequence(oracle):
    rng = np.random.default_rng(3)
    for q, n, depth in [(2, 5, 3), (3, 4, 2)]:
        pairs = [(s, s + 1) for layer in range(1, depth + 1) for s in range(1 if layer % 2 else 2, n, 2)]
        gates = [rng.normal(size=(q * q, q * q)) + 1j * rng.normal(size=(q * q, q * q)) for _ in pairs]
        psi = rand_state(q ** n, 9)
        ref = psi.copy()
        for (s1, s2), g in zip(pairs, gates):
            ref = _apply_2gate_numpy(ref, q, g, s1, s2)
        assert np.allclose(oracle.brick_wall(psi, q, depth, gates), ref, atol=1e-10)
