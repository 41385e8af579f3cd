"""MC_SRE, Mana (pure and mixed) and the adjoint on the GPU against the oracle.
MC chains run on identical injected proposal streams: the accepted X-strings must be
bit-exact and the estimate within 1e-10 relative."""
import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [3, 6, 11, 12, 15])
def test_mc_matches_oracle(ctx, hm, oracle, n):
    psi = rand_state(1 << n, 300 + n)
    nb, ns = 13, 150
    pd, rs = hm.proposal_stream(n, nb, ns, seed=123)
    m2, M2, M2ADD, P2, masks = ctx.mc_sre(psi, 2, nb, ns, pd, rs)
    om2, oM2, oM2ADD, oP2 = oracle.mc_sre(psi, 2, nb, ns, pd, rs)
    assert m2 == pytest.approx(om2, rel=1e-10)
    assert np.allclose(M2, oM2, rtol=1e-10) and np.allclose(M2ADD, oM2ADD, rtol=1e-10)
    assert np.allclose(P2, oP2, rtol=1e-10)
    for i in range(nb):
        _, om = oracle.mc_sre_beta(psi, 2, i / (nb - 1), pd[i], rs[i])
        assert int(masks[i]) == int(om[-1])


def test_mc_same_seed_reproducible(hm):
    # test/SRE_test.jl:183-211
    psi = hm.StateVec(rand_state(1 << 10, 9))
    a = hm.MC_SRE(psi, 2, Nbeta=13, Nsamples=300, seed=123)
    b = hm.MC_SRE(psi, 2, Nbeta=13, Nsamples=300, seed=123)
    assert a == b


def test_mc_generic_q(ctx, hm, oracle):
    n = 8
    psi = rand_state(1 << n, 8)
    pd, rs = hm.proposal_stream(n, 5, 80, seed=7)
    assert ctx.mc_sre(psi, 3.0, 5, 80, pd, rs)[0] == pytest.approx(oracle.mc_sre(psi, 3.0, 5, 80, pd, rs)[0],
                                                                  rel=1e-10)


@pytest.mark.parametrize("L", [1, 2, 3, 4, 5, 6, 7, 8])
def test_mana_pure_matches_oracle(ctx, oracle, L):
    psi = rand_state(3 ** L, 100 + L)
    assert ctx.mana_pure(psi) == pytest.approx(oracle.mana_pure(psi), rel=1e-10)


def test_mana_pure_basis_state_is_zero(hm):
    psi = np.zeros(3 ** 6, complex)
    psi[0] = 1
    assert abs(hm.Mana(hm.StateVec(psi, q=3))) < 1e-12


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_mana_mixed_matches_oracle(ctx, oracle, N):
    psi = rand_state(3 ** N, 200 + N)
    rho = np.outer(psi, psi.conj())
    assert ctx.mana_mixed(rho) == pytest.approx(oracle.mana_mixed(rho), rel=1e-10, abs=1e-12)


def test_mana_mixed_reduced_10_qutrits(hm, oracle):
    # 10 qutrits traced down to the 6 most significant: a 729 x 729 density matrix
    psi = hm.StateVec(rand_state(3 ** 10, 10), q=3)
    rho = hm.reduced_density_matrix(psi, 6, side="right")
    assert hm.Mana(rho) == pytest.approx(oracle.mana_mixed(rho.data), rel=1e-10)
    assert abs(hm.Mana(hm.DensityMatrix(np.eye(729) / 729, q=3))) < 1e-12


@pytest.mark.parametrize("n,q", [(1, 2), (3, 2), (6, 2), (9, 2), (11, 2), (12, 2), (13, 2), (14, 2), (12, 3)])
def test_grad_matches_oracle(ctx, oracle, n, q):
    psi = rand_state(1 << n, 500 + n)
    v, g = ctx.sre_grad(psi, q)
    ov, og = oracle.sre_grad(psi, q)
    assert v == pytest.approx(ov, rel=1e-10)
    assert np.max(np.abs(g - og)) <= 1e-10 * np.max(np.abs(og))


def test_grad_central_differences_n14(ctx, hm):
    n = 14
    psi = rand_state(1 << n, 14)
    v, g = ctx.sre_grad(psi, 2)
    rng = np.random.default_rng(64)
    h = 1e-6
    for r in rng.integers(0, 1 << n, size=32):
        for comp in (1.0, 1j):
            p, m = psi.copy(), psi.copy()
            p[r] += h * comp
            m[r] -= h * comp
            fd = (ctx.sre(p, (2.0,), hm.HM_FP64)[0][0] - ctx.sre(m, (2.0,), hm.HM_FP64)[0][0]) / (2 * h)
            an = g[r].real if comp == 1.0 else g[r].imag
            assert an == pytest.approx(fd, rel=1e-4, abs=1e-7)
