"""Exact SRE on the GPU against the oracle.  Tolerances: FP64 and the plain path
1e-10 relative (the stated FP64 bound; observed ~1e-15).  FP32 butterflies: 1e-6
relative or 1e-6 absolute, whichever is larger.  The absolute term covers values below
one: rounding each product f = conj(psi(r)) psi(r ^ x) to FP32 (2^-24 relative) already
moves SRE by about 1e-7 in absolute terms, so no relative bound holds as SRE -> 0 (an
n = 1 state with SRE_2 = 0.067 shows 1.2e-6 relative).  Full-size (n = 20) cases use
size-independent properties: analytic values of product and stabilizer states,
Parseval (lost_norm), and Gray sub-ranges checked against the oracle."""
import numpy as np
import pytest

from conftest import ghz, rand_state, t_state

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "plain": 1e-10, "fp32": 1e-6}
ABS = {"fp64": 0.0, "plain": 0.0, "fp32": 1e-6}


def close(ref, prec):
    return pytest.approx(ref, rel=TOL[prec], abs=ABS[prec])


@pytest.mark.parametrize("n", list(range(1, 17)))
def test_sre_matches_oracle(ctx, hm, oracle, n):
    psi = rand_state(1 << n, 100 + n)
    ref2, lost = oracle.sre(psi, 2)
    ref3, _ = oracle.sre(psi, 3)
    for prec in ("fp64", "fp32", "plain"):
        v, l = ctx.sre(psi, (2.0, 3.0), hm.PRECISIONS[prec])
        assert v[0] == close(ref2, prec), prec
        assert v[1] == close(ref3, prec), prec
        assert l < (1e-12 if prec != "fp32" else 1e-6)


@pytest.mark.parametrize("q", [1.0, 2.5, 4.0])
def test_generic_q(ctx, hm, oracle, q):
    for n in (5, 13):
        psi = rand_state(1 << n, 7 * n)
        ref, _ = oracle.sre(psi, q)
        v, _ = ctx.sre(psi, (q,), hm.HM_FP64)
        assert v[0] == pytest.approx(ref, rel=1e-10)


def test_public_api_matches_reference_semantics(hm, oracle, golden):
    for g in golden["sre"]:
        n, q = g["n"], g["q"]
        psi = (np.array(g["re"]) + 1j * np.array(g["im"])) if g["kind"] == "random" else (
            t_state(n) if g["kind"] == "t_state" else ghz(n))
        v, lost = hm.SRE(hm.StateVec(psi), q)
        assert v == pytest.approx(g["sre"], rel=1e-10, abs=1e-12)
        assert lost < 1e-12


@pytest.mark.parametrize("n", [18, 20])
def test_full_size_known_answers(ctx, hm, n):
    for prec in ("fp64", "fp32"):
        tol = TOL[prec]
        v, l = ctx.sre(t_state(n), (2.0, 3.0), hm.PRECISIONS[prec])
        assert v[0] == pytest.approx(n * np.log2(4 / 3), rel=tol)
        assert v[1] == pytest.approx(n * np.log2(8 / 5), rel=tol)
        v, l = ctx.sre(ghz(n), (2.0,), hm.PRECISIONS[prec])
        assert abs(v[0]) < 10 * tol
        v, l = ctx.sre(rand_state(1 << n, n), (2.0,), hm.PRECISIONS[prec])
        assert l < (1e-12 if prec == "fp64" else 1e-6)


@pytest.mark.parametrize("n", [17, 20])
def test_gray_subranges_match_oracle(ctx, hm, oracle, n):
    psi = rand_state(1 << n, n + 1)
    N = 1 << n
    for kb, ke in [(0, 24), (1000, 1030), (N // 2 + 5, N // 2 + 40), (N - 21, N)]:
        p2r, mr = oracle.sre_sums(psi, 2, kb + 1, ke)
        p2, m = ctx.sre_range(psi, kb, ke, (2.0,), hm.HM_FP64)
        assert p2.sum() == pytest.approx(p2r, rel=1e-12)
        assert m.sum() == pytest.approx(mr, rel=1e-12)


def test_range_additivity_and_determinism(ctx, hm):
    n = 15
    psi = rand_state(1 << n, 3)
    full_p2, full_m = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
    a = ctx.sre_range(psi, 0, 12345, (2.0,), hm.HM_FP64)
    b = ctx.sre_range(psi, 12345, 1 << n, (2.0,), hm.HM_FP64)
    s = hm.shard.dd_fold([a[1][0], b[1][0]])
    assert s[0] + s[1] == pytest.approx(full_m.sum(), rel=1e-15)
    again = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
    assert np.array_equal(again[1], full_m) and np.array_equal(again[0], full_p2)


def test_device_pointer_entry(ctx, hm, oracle):
    import torch
    n = 14
    psi = rand_state(1 << n, 5)
    t = torch.from_numpy(psi.view(np.float64).copy()).cuda()
    v, l = ctx.sre_dev(t.data_ptr(), n, (2.0,), hm.HM_FP64)
    assert v[0] == pytest.approx(oracle.sre(psi, 2)[0], rel=1e-10)
    with pytest.raises(hm.ArgumentError):
        ctx.sre_dev(t.data_ptr() + 8, n, (2.0,), hm.HM_FP64)  # not 16-byte aligned


def test_argument_errors(ctx, hm):
    with pytest.raises(hm.ArgumentError):
        ctx.sre(rand_state(8, 1), (0.5,), hm.HM_FP64)
    with pytest.raises(hm.ArgumentError):
        ctx.sre(rand_state(8, 1), (2.0,), 7)
    with pytest.raises(hm.ArgumentError):
        ctx.sre_range(rand_state(8, 1), 5, 9, (2.0,), hm.HM_FP64)
    with pytest.raises(hm.ArgumentError):
        ctx.sre(rand_state(8, 1), (2.0, 3.0, 2.0, 3.0, 2.0), hm.HM_FP64)


def test_gray_tables_bit_exact(ctx, oracle):
    for n in list(range(0, 13)) + [20]:
        c, f = ctx.gray_table(n)
        co, fo = oracle.gray_binary(n)
        assert np.array_equal(c, co) and np.array_equal(f, fo)
    for n, q in [(2, 3), (1, 4), (6, 3), (10, 3), (4, 5)]:
        x, f = ctx.gray_table_general(n, q)
        xo, fo = oracle.gray_general(n, q)
        assert np.array_equal(x, xo) and np.array_equal(f, fo)


def test_batched_matches_per_state(ctx, hm, oracle):
    rng = np.random.default_rng(512)
    ns = [int(v) for v in rng.integers(1, 16, size=24)]
    psis = [rand_state(1 << n, 10_000 + i) for i, n in enumerate(ns)]
    for prec in ("fp64", "fp32"):
        vals, lost = ctx.sre_batched(psis, (2.0, 3.0), hm.PRECISIONS[prec])
        for i, p in enumerate(psis):
            assert vals[i, 0] == close(oracle.sre(p, 2)[0], prec)
            assert vals[i, 1] == close(oracle.sre(p, 3)[0], prec)


def test_autotune_records_a_batch_size(ctx, hm, oracle):
    n = 13
    psi = rand_state(1 << n, 77)
    ref = oracle.sre(psi, 2)[0]
    for prec in ("fp64", "fp32"):
        x, us = ctx.autotune(n, hm.PRECISIONS[prec])
        assert x >= 1 and us > 0  # the stage kernels take any batch size, the queue a power of two
        eng, bx, cps = hm._native.autotune_choice(n, hm.PRECISIONS[prec])
        assert eng in (1, 2) and bx == x and cps in (0, 1)
        v, _ = ctx.sre(psi, (2.0,), hm.PRECISIONS[prec])  # runs with the tuned engine and batch size
        assert v[0] == close(ref, prec)
    with pytest.raises(hm.ArgumentError):
        ctx.autotune(11, hm.HM_FP64)


def test_split_gray_tables_match_oracle(ctx, oracle):
    """generate_binary_splitted / generate_general_splitted (src/Basis.jl:76-106, 206-250):
    every rank's slice bit-exact, and the slices concatenate to the whole table."""
    for n, P in [(5, 3), (10, 4), (11, 7), (3, 16)]:
        full, _ = ctx.gray_table(n)
        got = []
        for r in range(P):
            c, f, off = ctx.gray_table_split(n, 2, r, P)
            co, fo, oo = oracle.gray_binary_split(n, r, P)
            assert off == oo and np.array_equal(c, co) and np.array_equal(f, fo)
            got.append(c)
        assert np.array_equal(np.concatenate(got), full)
    for n, q, P in [(4, 3, 5), (6, 3, 4)]:
        xt, _ = ctx.gray_table_general(n, q)
        cols = []
        for r in range(P):
            x, f, off = ctx.gray_table_split(n, q, r, P)
            cols.append(x)
            if x.shape[1] > 1:
                assert np.array_equal(f, [int(np.argmax(x[:, j] != x[:, j + 1])) + 1 for j in range(x.shape[1] - 1)])
        assert np.array_equal(np.concatenate(cols, axis=1), xt)


@pytest.mark.parametrize("n,X", [(12, 1), (13, 3), (14, 1), (16, 6)])
def test_stage_ring_reuse_is_exact(ctx, hm, oracle, n, X):
    """Pass 2 drops each tile from L2 after reading it, and pass 1 of the stage after next
    rewrites the slot.  With tiny batches the stages are a few microseconds long, so a
    late drop would meet the new rows: every repetition must give the same bits, and the
    value must match the oracle."""
    N = hm._native
    psi = rand_state(1 << n, 900 + n)
    ref = oracle.sre(psi, 2)[0]
    N.set_param(N.HM_PARAM_ENGINE, 1)
    N.set_param(N.HM_PARAM_BATCH, X)
    try:
        first = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
        for _ in range(12):
            again = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
            assert np.array_equal(again[0], first[0]) and np.array_equal(again[1], first[1])
        v, _ = ctx.sre(psi, (2.0,), hm.HM_FP64)
        assert v[0] == close(ref, "fp64")
    finally:
        N.set_param(N.HM_PARAM_BATCH, 0)
        N.set_param(N.HM_PARAM_ENGINE, 0)


@pytest.mark.parametrize("n", [22, 23, 24])
def test_three_pass_sweep_matches_oracle(ctx, hm, oracle, n):
    """n = 22..24 run the three-pass stage kernels: Gray sub-ranges (x = 0 included, more
    batches than the three ring slots) against the oracle in FP64 and FP32, and against
    the plain multi-launch form; an odd batch size at n = 22."""
    psi = rand_state(1 << n, 2200 + n)
    N = 1 << n
    w = 9 if n == 22 else 5
    for kb, ke in [(0, w), (N // 2 + 3, N // 2 + 3 + w), (N - w, N)]:
        p2r, mr = oracle.sre_sums(psi, 2, kb + 1, ke)
        for prec, tol in (("fp64", 1e-12), ("fp32", 1e-6), ("plain", 1e-12)):
            p2, m = ctx.sre_range(psi, kb, ke, (2.0,), hm.PRECISIONS[prec])
            assert p2.sum() == pytest.approx(p2r, rel=tol), (kb, prec)
            assert m.sum() == pytest.approx(mr, rel=tol), (kb, prec)
    if n == 22:
        N_ = hm._native
        N_.set_param(N_.HM_PARAM_BATCH, 3)
        try:
            p2, m = ctx.sre_range(psi, 1000, 1011, (2.0, 3.0), hm.HM_FP64)
        finally:
            N_.set_param(N_.HM_PARAM_BATCH, 0)
        p2b, mb = ctx.sre_range(psi, 1000, 1011, (2.0, 3.0), hm.HM_FP64)
        assert p2.sum() == pytest.approx(p2b.sum(), rel=1e-13)
        assert np.allclose(m.sum(axis=1), mb.sum(axis=1), rtol=1e-13)
        p2r, mr = oracle.sre_sums(psi, 3, 1001, 1011)
        assert mb[1].sum() == pytest.approx(mr, rel=1e-12)
