"""CPU-only checks: the C ABI library loads and exports every entry point that
include/hadamag_b200.h declares; host-side containers, loaders and argument checks
behave like the reference's; compute calls fail loudly when no GPU is present."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, rand_state


def header_functions():
    src = open(os.path.join(ROOT, "include", "hadamag_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(hm):
    lib = hm._native.load_library()
    names = header_functions()
    assert "hm_sre" in names and "hm_mc_sre" in names and "hm_mana_pure" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(hm._native.EXPORTS)
    assert lib.hm_abi_version() == 1


def test_set_param_validation(hm):
    lib = hm._native.load_library()
    assert lib.hm_set_param(hm._native.HM_PARAM_BATCH, 5000) == hm._native.HM_ERR_ARG
    assert lib.hm_set_param(hm._native.HM_PARAM_BATCH, 3) == 0
    assert lib.hm_set_param(hm._native.HM_PARAM_RING, 1) == hm._native.HM_ERR_ARG
    assert lib.hm_set_param(99, 1) == hm._native.HM_ERR_ARG
    assert lib.hm_set_param(hm._native.HM_PARAM_BATCH, 4) == 0
    assert lib.hm_set_param(hm._native.HM_PARAM_BATCH, 0) == 0
    assert lib.hm_set_param(hm._native.HM_PARAM_ADJ_BATCH, 48) == hm._native.HM_ERR_ARG
    assert lib.hm_set_param(hm._native.HM_PARAM_ADJ_BATCH, 2048) == hm._native.HM_ERR_ARG
    assert lib.hm_set_param(hm._native.HM_PARAM_ADJ_BATCH, 64) == 0
    assert lib.hm_set_param(hm._native.HM_PARAM_ADJ_BATCH, 0) == 0


def test_null_context_rejected(hm):
    lib = hm._native.load_library()
    assert lib.hm_destroy(None) == hm._native.HM_ERR_ARG
    assert lib.hm_last_error(None) == b"null context"


def test_no_cpu_fallback_without_gpu(hm):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hm.HadaMAGError):
        hm.SRE(hm.StateVec(rand_state(8, 1)), 2)
    with pytest.raises(hm.HadaMAGError):
        hm.Mana(hm.StateVec(rand_state(9, 1), q=3))


def test_statevec_checks(hm):
    # src/State.jl:40-44 and test/State_test.jl:6-15
    sv = hm.StateVec(rand_state(8, 2))
    assert hm.qubits(sv) == 3 and hm.qudit_dim(sv) == 2 and len(sv) == 8
    with pytest.raises(hm.ArgumentError):
        hm.StateVec(np.ones(7))
    with pytest.raises(hm.ArgumentError):
        hm.StateVec(np.ones(8), q=3)
    assert hm.StateVec(np.ones(27), q=3).n == 3
    with pytest.raises(hm.ArgumentError):
        hm.DensityMatrix(np.ones((3, 2)), q=3)
    with pytest.raises(hm.ArgumentError):
        hm.DensityMatrix(np.eye(4), q=3)


def test_backend_selection(hm):
    assert isinstance(hm._choose_backend("b200"), hm.B200)
    assert isinstance(hm._choose_backend(":auto"), hm.B200)
    with pytest.raises(hm.ArgumentError):
        hm._choose_backend(":serial")
    with pytest.raises(hm.ArgumentError):
        hm.MC_SRE(hm.StateVec(rand_state(8, 1)), 2, Nbeta=12)


def test_load_state_roundtrip(hm, tmp_path):
    # test/State_test.jl:321-373
    data = np.array([0.1 + 0.2j, -0.3 + 0.4j, 0.5 - 0.6j, -0.7 - 0.8j])
    p = tmp_path / "s.npy"
    np.save(p, data)
    sv = hm.load_state(str(p))
    assert sv.n == 2 and sv.q == 2 and np.array_equal(sv.data, data)
    t = tmp_path / "s.txt"
    t.write_text("\n".join(f"{a.real} {a.imag}" for a in data))
    sv = hm.load_state(str(t))
    assert np.array_equal(sv.data, data)
    t.write_text("1 2 3")
    with pytest.raises(hm.ArgumentError):
        hm.load_state(str(t))


def test_oracle_reduced_density_matrix(oracle):
    # src/DensityMatrix.jl:113-117: rho_A[iA, jA] = sum_kB psi[iA dimB + kB] conj(psi[jA dimB + kB])
    psi = rand_state(3 ** 4, 3)
    rho = oracle.reduced_density_matrix(psi, 3, 2, side="right")
    dimA, dimB = 9, 9
    ref = np.zeros((dimA, dimA), complex)
    for i in range(dimA):
        for j in range(dimA):
            ref[i, j] = sum(psi[i * dimB + k] * np.conj(psi[j * dimB + k]) for k in range(dimB))
    assert np.allclose(rho, ref, atol=1e-15)
    rho_l = oracle.reduced_density_matrix(psi, 3, 2, side="left")
    ref_l = np.zeros((dimA, dimA), complex)
    for i in range(dimA):
        for j in range(dimA):
            ref_l[i, j] = sum(psi[i + dimA * k] * np.conj(psi[j + dimA * k]) for k in range(dimB))
    assert np.allclose(rho_l, ref_l, atol=1e-15)
    assert np.trace(rho).real == pytest.approx(1.0)


def test_proposal_stream(hm):
    # src/SRE.jl:142-170: tries in 1..9 single-site flips XOR-ed together
    pd, rs = hm.proposal_stream(6, 3, 500, seed=123)
    assert pd.shape == (3, 500) and rs.shape == (3, 500)
    assert np.all(pd < 64) and np.all((rs >= 0) & (rs < 1))
    pd2, rs2 = hm.proposal_stream(6, 3, 500, seed=123)
    assert np.array_equal(pd, pd2) and np.array_equal(rs, rs2)
    assert not np.array_equal(pd[0], pd[1])


def test_state_prep_argument_errors(hm):
    # host-side validation; no device work is reached
    with pytest.raises(hm.ArgumentError):
        hm.rand_haar(3, 2, q=4)
    with pytest.raises(hm.ArgumentError):
        hm.haar_random_unitary(5, 2)
    with pytest.raises(hm.ArgumentError):
        hm.reduced_density_matrix(hm.StateVec(rand_state(8, 1)), 4)
    with pytest.raises(hm.ArgumentError):
        hm.reduced_density_matrix(hm.StateVec(rand_state(8, 1)), 1, side="middle")
    assert hm.brick_wall_pairs(5, 3) == [(1, 2), (3, 4), (2, 3), (4, 5), (1, 2), (3, 4)]


def test_haar_random_unitary_is_unitary(hm):
    rng = np.random.default_rng(5)
    for q in (2, 3):
        U = hm.haar_random_unitary(q, 2, rng)
        assert U.shape == (q * q, q * q)
        assert np.allclose(U.conj().T @ U, np.eye(q * q), atol=1e-13)
