"""Range entry points that split MC_SRE and Mana across GPUs, on one GPU: a chain range of
hm_mc_sre_chains gives exactly the chains of the whole-grid call, and Mana X-string
ranges add up to the whole sum (and match the oracle on a prefix of the Gray order,
which covers the same X-strings)."""
import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [8, 13])
def test_mc_chain_ranges_equal_whole_grid(hm, ctx, n):
    nbeta, nsamples = 5, 64
    psi = rand_state(1 << n, 70 + n)
    pd, rs = hm.proposal_stream(n, nbeta, nsamples, seed=5)
    pd = np.asarray(pd, dtype=np.uint64).reshape(nbeta, nsamples)
    rs = np.asarray(rs, dtype=np.float64).reshape(nbeta, nsamples)
    m2, M2, M2ADD, P2, fm = ctx.mc_sre(psi, 2.0, nbeta, nsamples, pd.reshape(-1), rs.reshape(-1))
    parts = [(0, 2), (2, 3), (3, 5)]
    got = [ctx.mc_sre_chains(psi, 2.0, nbeta, cb, ce, nsamples, pd[cb:ce].reshape(-1), rs[cb:ce].reshape(-1))
           for cb, ce in parts]
    M2c = np.concatenate([g[0] for g in got])
    assert np.array_equal(M2c, M2)
    assert np.array_equal(np.concatenate([g[1] for g in got]), M2ADD)
    assert np.array_equal(np.concatenate([g[2] for g in got]), P2)
    assert np.array_equal(np.concatenate([g[3] for g in got]), fm)
    # the host combination of the gathered chains is the device's
    assert hm.shard.mc_combine(M2c, M2ADD) == pytest.approx(m2, rel=1e-14, abs=1e-15)
    with pytest.raises(hm.ArgumentError):
        ctx.mc_sre_chains(psi, 2.0, nbeta, 4, 6, nsamples, pd[:2].reshape(-1), rs[:2].reshape(-1))


@pytest.mark.parametrize("L", [3, 7, 10])
def test_mana_ranges_add_up(hm, ctx, oracle, L):
    psi = rand_state(3 ** L, 90 + L)
    D = 3 ** L
    whole = ctx.mana_pure(psi)
    cuts = [0, D // 7, D // 3 + 1, D - 5, D]
    parts = [ctx.mana_pure_range(psi, a, b) for a, b in zip(cuts[:-1], cuts[1:])]
    S = hm.shard.dd_fold(parts)
    assert np.log2(S[0] + S[1]) / np.log2(3.0) == pytest.approx(whole, rel=1e-14)
    j = L - 1  # the first 3^j Gray columns are the X-strings [0, 3^j)
    pre = ctx.mana_pure_range(psi, 0, 3 ** j)
    assert pre[0] + pre[1] == pytest.approx(oracle.mana_sum(psi, 1, 3 ** j), rel=1e-12)
    # world = 1 through the sharding helper
    assert hm.shard.mana_sharded(lambda a, b: ctx.mana_pure_range(psi, a, b), L, 0, 1) == pytest.approx(whole,
                                                                                                     rel=1e-14)
