"""hm_sre_noalloc: the exact-SRE entry point for callers that cannot allocate device
memory (code inside another framework's memory pool, plugins that must not grow the
device footprint).  It runs out of a fixed scratch array inside the library.  Checked
through the C ABI against the allocating entry point hm_sre and against the oracle on
the same states, two calls in a row (the second one starts from the scratch the first
one left).  Tolerance: 1e-10 relative, the FP64 bound of every exact-SRE test.  Named
test_zz_* so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from conftest import rand_state

pytestmark = pytest.mark.gpu

_dp = ctypes.POINTER(ctypes.c_double)


def _noalloc(lib, psi, qs):
    a = np.ascontiguousarray(psi, dtype=np.complex128)
    n = a.size.bit_length() - 1
    q = np.ascontiguousarray(qs, dtype=np.float64)
    out = np.zeros(q.size)
    lost = ctypes.c_double()
    rc = lib.hm_sre_noalloc(a.view(np.float64).ctypes.data_as(_dp), n, q.ctypes.data_as(_dp), q.size,
                            out.ctypes.data_as(_dp), ctypes.byref(lost), None)
    return rc, out, lost.value


@pytest.mark.parametrize("n", [1, 5, 9, 11])
def test_noalloc_matches_allocating_entry(hm, oracle, n):
    import torch
    torch.cuda.set_device(0)
    lib = hm._native.load_library()
    ctx = hm._native.default_context(0)
    for qs in ((2.0,), (2.0, 3.0), (2.5,)):
        psi = rand_state(1 << n, 900 + n)
        ref, ref_lost = ctx.sre(psi, qs, hm.HM_FP64)
        orc = [oracle.sre(psi, q)[0] for q in qs]
        for _ in range(2):
            rc, out, lost = _noalloc(lib, psi, qs)
            assert rc == 0
            assert np.allclose(out, ref, rtol=1e-10, atol=1e-12)
            assert np.allclose(out, orc, rtol=1e-10, atol=1e-12)
            assert lost == pytest.approx(ref_lost, abs=1e-12)


def test_noalloc_rejects_sizes_beyond_its_maximum(hm):
    lib = hm._native.load_library()
    rc, _, _ = _noalloc(lib, rand_state(1 << 12, 1), (2.0,))
    assert rc == hm._native.HM_ERR_SIZE
