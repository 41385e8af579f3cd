"""The BASELINE-size configurations on the GPU against the oracle.

Tolerances: FP64 1e-10 relative (the stated FP64 bound); FP32 butterflies 1e-6 relative
or absolute, whichever is larger (the stated FP32 bound; see test_gpu_sre.py); MC masks
bit-exact; the adjoint's central differences 1e-4 relative or 1e-7 absolute (the step
1e-6 leaves about 1e-8 of rounding noise in a difference of two SRE values near 18).

Heavy oracle runs come from committed fixtures made by the oracle in this repository
(tests/golden/gen_n20.py, tests/golden/gen_large.py); light ones run here.
"""
import json
import os

import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"fixture {name} missing: run tests/golden/gen_n20.py / gen_large.py")
    with open(path) as f:
        return json.load(f)


def _dd(x):
    return float(x[0]) + float(x[1])


# ------------------------------------------------------------------ exact SRE, N = 20

@pytest.fixture(scope="module")
def n20():
    fx = _fixture("n20_seed20.json")
    psi = rand_state(1 << 20, 20)  # default_rng(20), the bench's state
    return fx, psi


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_n20_seed20_q2_q3_matches_oracle_fixture(ctx, hm, n20, prec):
    fx, psi = n20
    p2, m = ctx.sre_range(psi, 0, 1 << 20, (2.0, 3.0), hm.PRECISIONS[prec])
    dim = float(1 << 20)
    for i, q in enumerate((2.0, 3.0)):
        j = fx["qs"].index(q)
        val = -np.log2((m[i, 0] + m[i, 1]) / dim)
        if prec == "fp64":
            assert _dd(m[i]) == pytest.approx(_dd(fx["m_dd"][j]), rel=1e-10)
            assert val == pytest.approx(fx["sre"][j], rel=1e-10)
        else:
            assert val == pytest.approx(fx["sre"][j], rel=1e-6, abs=1e-6)
    assert _dd(p2) == pytest.approx(_dd(fx["p2_dd"]), rel=1e-10 if prec == "fp64" else 1e-6)


def test_n20_public_api_value(hm, n20):
    fx, psi = n20
    v, lost = hm.SRE(hm.StateVec(psi), 2)
    assert v == pytest.approx(fx["sre"][0], rel=1e-10)
    assert lost == pytest.approx(fx["lost_norm"], abs=1e-12)


def test_n20_gray_subranges_match_oracle_fixture(ctx, hm, n20):
    fx, psi = n20
    for sub in fx["subranges"]:
        p2, m = ctx.sre_range(psi, sub["k_begin"], sub["k_end"], (2.0, 3.0), hm.HM_FP64)
        assert _dd(p2) == pytest.approx(_dd(sub["p2"]), rel=1e-12)
        for i in range(2):
            assert _dd(m[i]) == pytest.approx(_dd(sub["m"][i]), rel=1e-12)


# ------------------------------------------------------------------ Gray sub-ranges, n = 18, 19, 21

@pytest.mark.parametrize("n", [18, 19, 21])
def test_gray_subranges_large_n_match_oracle(ctx, hm, oracle, n):
    """Exercises the stage kernels at HI = n - 11 = 7, 8, 10 (and the relabelled copies
    for x < 2^10) against the oracle's fast path."""
    psi = rand_state(1 << n, n + 1)
    N = 1 << n
    for kb, ke in [(0, 40), (1000, 1060), (N // 2 - 17, N // 2 + 17), (N - 24, N)]:
        p2r, mr = oracle.sre_sums_fast(psi, (2.0, 3.0), kb + 1, ke)
        for prec, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
            p2, m = ctx.sre_range(psi, kb, ke, (2.0, 3.0), hm.PRECISIONS[prec])
            assert _dd(p2) == pytest.approx(_dd(p2r), rel=tol)
            for i in range(2):
                assert _dd(m[i]) == pytest.approx(_dd(mr[i]), rel=tol)


# ------------------------------------------------------------------ MC_SRE, N = 20

def test_mc_n20_matches_oracle(ctx, hm, oracle, n20):
    """C2-MC's kernels (k_mc_p1 / k_mc_p2 at HI = 9) on 13 chains x 150 steps of an
    injected stream: the final X-string of every chain bit-exact, m2 within 1e-10."""
    _, psi = n20
    n, nb, ns = 20, 13, 150
    pd, rs = hm.proposal_stream(n, nb, ns, seed=123)
    m2, M2, M2ADD, P2, masks = ctx.mc_sre(psi, 2, nb, ns, pd, rs)
    om2, oM2, oM2ADD, oP2 = oracle.mc_sre(psi, 2, nb, ns, pd, rs)
    assert m2 == pytest.approx(om2, rel=1e-10)
    assert np.allclose(M2, oM2, rtol=1e-10) and np.allclose(P2, oP2, rtol=1e-10)
    assert np.allclose(M2ADD, oM2ADD, rtol=1e-10)
    for i in (0, 6, 12):
        _, om = oracle.mc_sre_beta(psi, 2, i / (nb - 1), pd[i], rs[i])
        assert int(masks[i]) == int(om[-1])


def test_mc_more_than_31_chains(ctx, hm, oracle):
    """The reference takes any odd number of beta points (src/Backends/Threads.jl:169)."""
    n, nb, ns = 9, 41, 30
    psi = rand_state(1 << n, 41)
    pd, rs = hm.proposal_stream(n, nb, ns, seed=5)
    m2, M2, _, _, masks = ctx.mc_sre(psi, 2, nb, ns, pd, rs)
    om2, oM2, _, _ = oracle.mc_sre(psi, 2, nb, ns, pd, rs)
    assert m2 == pytest.approx(om2, rel=1e-10)
    assert np.allclose(M2, oM2, rtol=1e-10)
    n = 13
    psi = rand_state(1 << n, 13)
    pd, rs = hm.proposal_stream(n, 33, 12, seed=6)
    assert ctx.mc_sre(psi, 2, 33, 12, pd, rs)[0] == pytest.approx(oracle.mc_sre(psi, 2, 33, 12, pd, rs)[0],
                                                                  rel=1e-10)


# ------------------------------------------------------------------ adjoint, N = 16 and 18

def test_grad_n16_matches_oracle(ctx, oracle):
    n = 16
    psi = rand_state(1 << n, 500 + n)
    v, g = ctx.sre_grad(psi, 2)
    ov, og = oracle.sre_grad(psi, 2)
    assert v == pytest.approx(ov, rel=1e-10)
    assert np.max(np.abs(g - og)) <= 1e-10 * np.max(np.abs(og))


@pytest.fixture(scope="module")
def grad18(ctx):
    fx = _fixture("grad_n18_seed18.json")
    psi = rand_state(1 << 18, 18)
    v, g = ctx.sre_grad(psi, 2)
    return fx, psi, v, g


def test_grad_n18_matches_oracle_fixture(grad18):
    """BASELINE C4 at N = 18 (the X = 512 batch and the HI = 7 stage kernels): 64 seeded
    coordinates and 4 seeded projections of the oracle's gradient."""
    fx, psi, v, g = grad18
    assert v == pytest.approx(fx["sre"], rel=1e-10)
    idx = np.array(fx["idx"])
    og = np.array(fx["g_re"]) + 1j * np.array(fx["g_im"])
    scale = fx["max_abs"]
    assert np.max(np.abs(g[idx] - og)) <= 1e-10 * scale
    for k, proj in enumerate(fx["proj"]):
        w = np.random.default_rng(1000 + k).normal(size=(1 << 18, 2))
        got = float(np.sum(w[:, 0] * g.real + w[:, 1] * g.imag))
        assert got == pytest.approx(proj, rel=1e-9, abs=1e-10 * scale * 512)


def test_grad_n18_central_differences_64_coordinates(ctx, hm, grad18):
    """BASELINE C4: central differences, step 1e-6, on 64 seeded real coordinates."""
    _, psi, _, g = grad18
    n = 18
    rng = np.random.default_rng(64)
    idx = rng.integers(0, 1 << n, size=64)
    comps = rng.integers(0, 2, size=64)
    h = 1e-6
    for r, c in zip(idx, comps):
        step = h if c == 0 else 1j * h
        p, m = psi.copy(), psi.copy()
        p[r] += step
        m[r] -= step
        fd = (ctx.sre(p, (2.0,), hm.HM_FP64)[0][0] - ctx.sre(m, (2.0,), hm.HM_FP64)[0][0]) / (2 * h)
        an = g[r].real if c == 0 else g[r].imag
        assert an == pytest.approx(fd, rel=1e-4, abs=1e-7)


# ------------------------------------------------------------------ Mana, L = 10 and 11

@pytest.mark.parametrize("L", [10, 11])
def test_mana_pure_full_matches_oracle_fixture(ctx, L):
    fx = _fixture("mana_pure_L10_L11.json")[str(L)]
    psi = rand_state(3 ** L, L)
    assert ctx.mana_pure(psi) == pytest.approx(fx["mana"], rel=1e-10)
    s = ctx.mana_pure_range(psi, 0, 3 ** L)
    assert _dd(s) == pytest.approx(fx["sum"], rel=1e-10)


def test_mana_pure_L12_runs_and_matches_range_sum(ctx):
    """The largest supported size: the full call equals the sum of two range calls."""
    L = 12
    psi = rand_state(3 ** L, L)
    full = ctx.mana_pure(psi)
    a = ctx.mana_pure_range(psi, 0, 3 ** 11)
    b = ctx.mana_pure_range(psi, 3 ** 11, 3 ** L)
    assert full == pytest.approx(np.log2(_dd(a) + _dd(b)) / np.log2(3), rel=1e-12)
