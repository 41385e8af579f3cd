"""The persistent queue sweep (csrc/sweep_queue.cuh): one launch over the work units of one
or many states, with batch counters in place of kernel boundaries.

Checked against the oracle (FP64 1e-10 relative, FP32 1e-6 relative or absolute), against
the stage-kernel sweep on the same state (1e-13), under every knob of the queue (slots,
claim size, CTAs per SM, batch size: the sums may only differ by double-double rounding),
on batches of states of mixed sizes, and for the status of a wait that gives up."""
import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu


@pytest.fixture
def knobs(hm):
    set_param = hm._native.set_param
    N = hm._native
    yield set_param
    for p in (N.HM_PARAM_ENGINE, N.HM_PARAM_QUEUE_SLOTS, N.HM_PARAM_QUEUE_SLOT_MIB, N.HM_PARAM_QUEUE_CHUNK,
              N.HM_PARAM_QUEUE_CTAS, N.HM_PARAM_BATCH, N.HM_PARAM_QUEUE_STALL_TEST, N.HM_PARAM_QUEUE_LEAD,
              N.HM_PARAM_BATCH_SPLIT_N):
        set_param(p, 0)


def _dd(x):
    return float(x[0]) + float(x[1])


@pytest.mark.parametrize("n", [12, 13, 14, 15, 16])
def test_queue_matches_oracle(ctx, hm, oracle, knobs, n):
    knobs(hm._native.HM_PARAM_ENGINE, 2)
    psi = rand_state(1 << n, 700 + n)
    r2 = oracle.sre(psi, 2)[0]
    r3 = oracle.sre(psi, 3)[0]
    for prec, tol, atol in (("fp64", 1e-10, 0.0), ("fp32", 1e-6, 1e-6)):
        v, lost = ctx.sre(psi, (2.0, 3.0), hm.PRECISIONS[prec])
        assert v[0] == pytest.approx(r2, rel=tol, abs=atol)
        assert v[1] == pytest.approx(r3, rel=tol, abs=atol)
        assert lost < (1e-12 if prec == "fp64" else 1e-6)


@pytest.mark.parametrize("n", [17, 19, 20, 21])
def test_queue_matches_stage_kernels(ctx, hm, knobs, n):
    psi = rand_state(1 << n, 800 + n)
    N = 1 << n
    ranges = [(0, 3000), (N // 3, N // 3 + 2000)] if n >= 20 else [(0, N)]
    for kb, ke in ranges:
        knobs(hm._native.HM_PARAM_ENGINE, 1)
        p2s, ms = ctx.sre_range(psi, kb, ke, (2.0, 3.0), hm.HM_FP64)
        knobs(hm._native.HM_PARAM_ENGINE, 2)
        p2q, mq = ctx.sre_range(psi, kb, ke, (2.0, 3.0), hm.HM_FP64)
        assert _dd(p2q) == pytest.approx(_dd(p2s), rel=1e-13)
        for i in range(2):
            assert _dd(mq[i]) == pytest.approx(_dd(ms[i]), rel=1e-13)


def test_queue_knobs_do_not_change_the_sums(ctx, hm, knobs):
    N = hm._native
    knobs(N.HM_PARAM_ENGINE, 2)
    n = 15
    psi = rand_state(1 << n, 77)
    base = ctx.sre_range(psi, 0, 1 << n, (2.0, 3.0), hm.HM_FP64)
    for param, val in ((N.HM_PARAM_QUEUE_SLOTS, 2), (N.HM_PARAM_QUEUE_SLOTS, 9), (N.HM_PARAM_QUEUE_CHUNK, 5),
                       (N.HM_PARAM_QUEUE_CTAS, 1), (N.HM_PARAM_BATCH, 1), (N.HM_PARAM_BATCH, 64), (N.HM_PARAM_BATCH, 6),
                       (N.HM_PARAM_QUEUE_SLOT_MIB, 1), (N.HM_PARAM_QUEUE_LEAD, 1), (N.HM_PARAM_QUEUE_LEAD, 5)):
        knobs(param, val)
        p2, m = ctx.sre_range(psi, 0, 1 << n, (2.0, 3.0), hm.HM_FP64)
        knobs(param, 0)
        assert _dd(p2) == pytest.approx(_dd(base[0]), rel=1e-14), (param, val)
        for i in range(2):
            assert _dd(m[i]) == pytest.approx(_dd(base[1][i]), rel=1e-14), (param, val)


def test_queue_repeatable(ctx, hm, knobs):
    knobs(hm._native.HM_PARAM_ENGINE, 2)
    n = 16
    psi = rand_state(1 << n, 5)
    a = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
    b = ctx.sre_range(psi, 0, 1 << n, (2.0,), hm.HM_FP64)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("split", [22, 0])
def test_batched_mixed_sizes_matches_per_state(ctx, hm, oracle, knobs, split):
    """The C3 shape on a smaller scale: n drawn from 8..18, q = 2 and 3; every state in one
    queue launch (split 22), or the default split (n >= 15 one state per call)."""
    knobs(hm._native.HM_PARAM_BATCH_SPLIT_N, split)
    rng = np.random.default_rng(512)
    ns = [int(v) for v in rng.integers(8, 19, size=40)]
    psis = [rand_state(1 << n, 10_000 + i) for i, n in enumerate(ns)]
    for prec, tol, atol in (("fp64", 1e-10, 0.0), ("fp32", 1e-6, 1e-6)):
        vals, lost = ctx.sre_batched(psis, (2.0, 3.0), hm.PRECISIONS[prec])
        if split == 22:
            assert ctx.last_launch_count() <= 6  # queue kernel + fold (+ the FP64 x = 0 launch in FP32)
        for i, p in enumerate(psis):
            ref, rlost = ctx.sre(p, (2.0, 3.0), hm.HM_FP64)
            assert vals[i, 0] == pytest.approx(ref[0], rel=tol, abs=atol)
            assert vals[i, 1] == pytest.approx(ref[1], rel=tol, abs=atol)
        for i in (0, 7):
            if ns[i] <= 16:
                assert vals[i, 0] == pytest.approx(oracle.sre(psis[i], 2)[0], rel=tol, abs=atol)


def test_queue_slot_reuse_across_states(ctx, hm, knobs):
    """Batches of different unit counts in one launch.  Large slots (256 MiB, three of
    them): an n = 12 state's single batch holds all its 4096 X-strings (8192 units per
    pass) while the n >= 13 states fill the slot (16384 units), so the first pass-1 units
    of an n = 12 state reuse the slot of a larger state's batch, and must wait for all of
    that batch's pass-2 units, not for as many as their own batch has.  Then FP32, whose
    x = 0 transforms run as one-X-string batches of 2^(n - 11) units.  Every repetition
    must give the per-state values."""
    N = hm._native
    knobs(N.HM_PARAM_BATCH_SPLIT_N, 22)
    knobs(N.HM_PARAM_QUEUE_SLOT_MIB, 256)
    knobs(N.HM_PARAM_QUEUE_SLOTS, 3)
    knobs(N.HM_PARAM_QUEUE_LEAD, 1)
    ns = [16, 12, 13, 12, 14, 12, 12, 13, 12]
    psis = [rand_state(1 << n, 4242 + i) for i, n in enumerate(ns)]
    refs = [ctx.sre(p, (2.0,), hm.HM_FP64)[0][0] for p in psis]
    for _ in range(6):
        vals, _ = ctx.sre_batched(psis, (2.0,), hm.HM_FP64)
        for i in range(len(ns)):
            assert vals[i, 0] == pytest.approx(refs[i], rel=1e-12), (i, ns[i])
    # FP32: every state's x = 0 transform runs as a one-X-string batch of its own in one
    # FP64 launch, so consecutive batches there have 2^(n - 11) units each
    for p in (N.HM_PARAM_QUEUE_SLOT_MIB, N.HM_PARAM_QUEUE_SLOTS, N.HM_PARAM_QUEUE_LEAD):
        knobs(p, 0)
    ns = [18, 17, 16, 15, 14, 13, 12, 12, 12, 12, 13, 12]
    psis = [rand_state(1 << n, 4343 + i) for i, n in enumerate(ns)]
    refs = [ctx.sre(p, (2.0,), hm.HM_FP64)[0][0] for p in psis]
    for _ in range(6):
        vals, _ = ctx.sre_batched(psis, (2.0,), hm.HM_FP32)
        for i in range(len(ns)):
            assert vals[i, 0] == pytest.approx(refs[i], rel=1e-6), (i, ns[i])


def test_batched_generic_q_and_tiny_states(ctx, hm, oracle):
    ns = [1, 2, 5, 11, 12, 13, 3]
    psis = [rand_state(1 << n, 40 + i) for i, n in enumerate(ns)]
    vals, _ = ctx.sre_batched(psis, (2.5, 4.0), hm.HM_FP64)
    for i, p in enumerate(psis):
        assert vals[i, 0] == pytest.approx(oracle.sre(p, 2.5)[0], rel=1e-10)
        assert vals[i, 1] == pytest.approx(oracle.sre(p, 4.0)[0], rel=1e-10)


def test_queue_wait_that_gives_up_reports_timeout(ctx, hm, knobs):
    """A pass-2 wait on a count nothing reaches gives up after its poll limit: the call
    returns HM_ERR_TIMEOUT and the context keeps working."""
    n = 13
    psi = rand_state(1 << n, 3)
    knobs(hm._native.HM_PARAM_ENGINE, 2)
    knobs(hm._native.HM_PARAM_QUEUE_STALL_TEST, 1)
    with pytest.raises(hm.HadaMAGError, match="gave up"):
        ctx.sre(psi, (2.0,), hm.HM_FP64)
    knobs(hm._native.HM_PARAM_QUEUE_STALL_TEST, 0)
    v, _ = ctx.sre(psi, (2.0,), hm.HM_FP64)
    knobs(hm._native.HM_PARAM_ENGINE, 1)
    w, _ = ctx.sre(psi, (2.0,), hm.HM_FP64)
    assert v[0] == pytest.approx(w[0], rel=1e-13)


def test_sre_multi_matches_single_device(hm, ctx):
    """hm_sre_multi on one GPU listed one, two and three times (separate contexts, run one
    after another on the device's thread): the range split and the double-double combine
    give the single-call value."""
    n = 16
    psi = rand_state(1 << n, 61)
    ref, rlost = ctx.sre(psi, (2.0, 3.0), hm.HM_FP64)
    for devs in ([0], [0, 0], [0, 0, 0]):
        v, lost = hm._native.sre_multi(devs, psi, (2.0, 3.0), hm.HM_FP64)
        assert np.allclose(v, ref, rtol=1e-13)
        assert lost == pytest.approx(rlost, abs=1e-14)
    p2, m = hm._native.sre_range_multi([0, 0], psi, 1000, 5000, (2.0,), hm.HM_FP64)
    r2, rm = ctx.sre_range(psi, 1000, 5000, (2.0,), hm.HM_FP64)
    assert _dd(p2) == pytest.approx(_dd(r2), rel=1e-14) and _dd(m[0]) == pytest.approx(_dd(rm[0]), rel=1e-14)
    v, _ = hm.SRE(hm.StateVec(psi), 2, backend=hm.B200(devices=[0, 0]))
    assert v == pytest.approx(ref[0], rel=1e-13)
    with pytest.raises(hm.ArgumentError):
        hm._native.sre_multi([], psi, (2.0,), hm.HM_FP64)
    hm._native.multi_release()
