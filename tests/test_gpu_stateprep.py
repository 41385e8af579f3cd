"""State preparation on the GPU (two-site gates, brick walls, reduced density matrices)
against the oracle (oracle/hm_oracle.c or_apply_2gate, or_brick_wall,
or_reduced_density_matrix, which restate src/State.jl:254-345, 146-221 and
src/DensityMatrix.jl:94-123).  Tolerance 1e-12 absolute on unit-norm states: the device
sums the same products in another order (fused multiply-adds)."""
import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu


def _rand_gate(rng, q):
    return rng.normal(size=(q * q, q * q)) + 1j * rng.normal(size=(q * q, q * q))


@pytest.mark.parametrize("q,n", [(2, 2), (2, 5), (2, 11), (3, 2), (3, 4), (3, 7)])
def test_apply_2gate_matches_oracle(ctx, oracle, q, n):
    rng = np.random.default_rng(100 * q + n)
    psi = rand_state(q ** n, n)
    pairs = [(a, b) for a in range(1, n + 1) for b in range(1, n + 1) if a != b]
    if len(pairs) > 12:
        pairs = [pairs[i] for i in rng.choice(len(pairs), 12, replace=False)] + [(1, n), (n, 1), (1, 2)]
    for s1, s2 in pairs:
        g = _rand_gate(rng, q)
        out = ctx.apply_2gate(psi, q, g, s1, s2)
        assert np.max(np.abs(out - oracle.apply_2gate(psi, q, g, s1, s2))) < 1e-12, (s1, s2)


@pytest.mark.parametrize("q,n,depth", [(2, 12, 6), (2, 3, 5), (3, 7, 4)])
def test_brick_wall_matches_oracle(hm, ctx, oracle, q, n, depth):
    rng = np.random.default_rng(7 + n)
    gates = [hm.haar_random_unitary(q, 2, rng) for _ in hm.brick_wall_pairs(n, depth)]
    psi = rand_state(q ** n, 2 * n)
    out = ctx.brick_wall(psi, q, depth, gates)
    assert np.max(np.abs(out - oracle.brick_wall(psi, q, depth, gates))) < 1e-12
    assert np.linalg.norm(out) == pytest.approx(1.0, abs=1e-12)


def test_rand_haar_full_size_norm(hm):
    # size-independent property at n = 20: unitary gates keep the norm
    sv = hm.rand_haar(20, 10, rng=np.random.default_rng(20))
    assert np.linalg.norm(sv.data) == pytest.approx(1.0, abs=1e-11)
    sv3 = hm.rand_haar(10, 6, q=3, rng=np.random.default_rng(10))
    assert np.linalg.norm(sv3.data) == pytest.approx(1.0, abs=1e-12)


def test_rand_cliff_is_a_stabilizer_state(hm):
    # every gate of the list is Clifford, so SRE_2 = 0 (known answer)
    for seed in range(3):
        sv = hm.rand_cliff(10, depth=6, rng=np.random.default_rng(seed))
        v, lost = hm.SRE(sv, 2)
        assert abs(v) < 1e-9 and lost < 1e-12


@pytest.mark.parametrize("q,n,NA", [(2, 12, 0), (2, 12, 3), (2, 12, 6), (2, 12, 12), (2, 9, 8), (3, 10, 6),
                                    (3, 6, 1), (3, 5, 5)])
def test_reduced_density_matrix_matches_oracle(ctx, oracle, q, n, NA):
    psi = rand_state(q ** n, 40 + n + NA)
    for side in ("left", "right"):
        rho = ctx.reduced_density_matrix(psi, q, NA, side)
        ref = oracle.reduced_density_matrix(psi, q, NA, side)
        assert np.max(np.abs(rho - ref)) < 1e-12, side


def test_reduced_density_matrix_full_size_properties(ctx):
    psi = rand_state(1 << 20, 99)
    for NA, side in ((10, "right"), (2, "left"), (14, "left")):
        rho = ctx.reduced_density_matrix(psi, 2, NA, side)
        assert np.trace(rho).real == pytest.approx(1.0, abs=1e-12)
        assert np.max(np.abs(rho - rho.conj().T)) < 1e-14
    # a product state |a> (x) |b>: rho of either block is |a><a| or |b><b|
    a = rand_state(1 << 6, 1)
    b = rand_state(1 << 8, 2)
    prod = np.kron(b, a)  # sites 1..6 hold a (least significant), 7..14 hold b
    assert np.allclose(ctx.reduced_density_matrix(prod, 2, 6, "left"), np.outer(a, a.conj()), atol=1e-14)
    assert np.allclose(ctx.reduced_density_matrix(prod, 2, 8, "right"), np.outer(b, b.conj()), atol=1e-14)


def test_haar_qutrit_pipeline_mana(hm, oracle):
    # rand_haar (10 qutrits) -> reduced density matrix of 6 -> Mana, all on the GPU,
    # against the oracle's density matrix and mixed-state Mana
    sv = hm.rand_haar(10, 4, q=3, rng=np.random.default_rng(6))
    rho = hm.reduced_density_matrix(sv, 6, side="right")
    ref = oracle.reduced_density_matrix(sv.data, 3, 6, "right")
    assert np.max(np.abs(rho.data - ref)) < 1e-13
    assert hm.Mana(rho) == pytest.approx(oracle.mana_mixed(ref), rel=1e-10)


def test_state_prep_argument_errors(hm, ctx):
    psi = rand_state(1 << 4, 1)
    g = np.eye(4)
    with pytest.raises(hm.ArgumentError):
        ctx.apply_2gate(psi, 2, g, 2, 2)  # same site twice
    with pytest.raises(hm.ArgumentError):
        ctx.apply_2gate(psi, 2, g, 1, 5)  # site outside [1, n]
    with pytest.raises(hm.ArgumentError):
        ctx.apply_2gate(psi, 2, np.eye(9), 1, 2)  # gate of the wrong size
    with pytest.raises(hm.ArgumentError):
        ctx.brick_wall(psi, 2, 3, [g] * 3)  # depth 3 on 4 sites takes 5 gates
    with pytest.raises(hm.ArgumentError):
        ctx.reduced_density_matrix(psi, 2, 5)
    with pytest.raises(hm.ArgumentError):
        ctx.apply_2gate(rand_state(27, 1), 4, np.eye(16), 1, 2)
    # the state is unchanged by a rejected call, and an identity brick wall is a no-op
    out = ctx.brick_wall(psi, 2, 3, [g] * 5)
    assert np.array_equal(out, psi)


def test_mana_range_argument_errors(hm, ctx):
    psi = rand_state(3 ** 4, 2)
    for a, b in ((0, 0), (5, 3), (-1, 4), (0, 82)):
        with pytest.raises(hm.ArgumentError):
            ctx.mana_pure_range(psi, a, b)


def test_load_state_pinned_matches_numpy(hm, tmp_path):
    """hm_load_state reads .npy and text files into page-locked memory with the same
    amplitudes numpy reads; the buffer is registered with CUDA as host-pinned."""
    psi = rand_state(1 << 9, 9)
    p = tmp_path / "s.npy"
    np.save(p, psi)
    s = hm.load_state(str(p))
    assert np.array_equal(s.data, psi) and s.n == 9
    import torch
    assert torch.from_numpy(s.data.view(np.float64)).is_pinned()
    t = tmp_path / "s.txt"
    t.write_text("\n".join(f"{float(z.real)!r} {float(z.imag)!r}" for z in psi))
    assert np.array_equal(hm.load_state(str(t)).data, psi)
    np.save(tmp_path / "r.npy", psi.real)
    assert np.array_equal(hm.load_state(str(tmp_path / "r.npy")).data, psi.real.astype(complex))
    np.save(tmp_path / "bad.npy", psi[:100])
    with pytest.raises(hm.ArgumentError):
        hm.load_state(str(tmp_path / "bad.npy"))
    with pytest.raises(hm.ArgumentError):
        hm.load_state(str(tmp_path / "s.jld2"))
    v, _ = hm.SRE(s, 2)
    assert v == pytest.approx(hm.SRE(hm.StateVec(psi), 2)[0], rel=1e-15)
