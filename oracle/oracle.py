"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: this module is the parity checker and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs import it; the product path never does.

Every function mirrors a function of hm_oracle.c, which cites the HadaMAG.jl
source (file:line) it restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build(force=False):
    """Compile liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "hm_oracle.c"))
    ):
        subprocess.run(["make", "-B" if force else "-s", "-C", _HERE], check=True,
                       env={k: v for k, v in os.environ.items() if k not in ("CC", "CFLAGS")})


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i, d = ctypes.c_int, ctypes.c_double
        L.or_gray_binary.argtypes = [i, _u64p, _i64p]
        L.or_gray_binary_split.argtypes = [i, i, i, _u64p, _i64p, _i64p]
        L.or_gray_general.argtypes = [i, i, _i64p, _i64p]
        L.or_partition_counts.argtypes = [ctypes.c_int64, i, _i64p, _i64p]
        L.or_fwht.argtypes = [_dp, i]
        L.or_fht_qutrit.argtypes = [_dp, ctypes.c_int64]
        L.or_sre_sums.argtypes = [_dp, i, d, ctypes.c_int64, ctypes.c_int64, i, _dp, _dp]
        L.or_sre_sums_fast.argtypes = [_dp, i, _dp, i, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, i, _dp]
        L.or_sre.argtypes = [_dp, i, d, i, _dp, _dp]
        L.or_naive_sre.argtypes = [_dp, i, i, i, _dp]
        L.or_mc_sre_beta.argtypes = [_dp, i, d, i, d, _u64p, _dp, _dp, _u64p]
        L.or_simpson_uniform.argtypes = [_dp, _dp, i]
        L.or_simpson_uniform.restype = d
        L.or_mc_sre.argtypes = [_dp, i, d, i, i, _u64p, _dp, i, _dp, _dp, _dp, _dp]
        L.or_mana_sum.argtypes = [_dp, i, ctypes.c_int64, ctypes.c_int64, i, _dp]
        L.or_mana_pure.argtypes = [_dp, i, i, _dp]
        L.or_single_qutrit_M.argtypes = [_dp]
        L.or_mana_mixed.argtypes = [_dp, i, _dp, _dp]
        L.or_sre_grad.argtypes = [_dp, i, d, i, _dp, _dp]
        L.or_apply_2gate.argtypes = [_dp, i, i, _dp, i, i]
        L.or_brick_wall.argtypes = [_dp, i, i, i, _dp, i]
        L.or_reduced_density_matrix.argtypes = [_dp, i, i, i, i, _dp]
        _lib = L
    return _lib


def _cplx(psi):
    a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128))
    return a, a.view(np.float64).ctypes.data_as(_dp)


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed with status {rc}")


def nthreads_default():
    return os.cpu_count() or 1


def gray_binary(n):
    N = 1 << n
    codes = np.zeros(N, dtype=np.uint64)
    flips = np.zeros(max(N - 1, 1), dtype=np.int64)
    _check(lib().or_gray_binary(n, codes.ctypes.data_as(_u64p), flips.ctypes.data_as(_i64p)), "gray_binary")
    return codes, flips[: N - 1]


def gray_binary_split(n, rank, P):
    N = 1 << n
    codes = np.zeros(N, dtype=np.uint64)
    flips = np.zeros(N, dtype=np.int64)
    off = ctypes.c_int64(0)
    _check(lib().or_gray_binary_split(n, rank, P, codes.ctypes.data_as(_u64p), flips.ctypes.data_as(_i64p),
                                      ctypes.byref(off)), "gray_binary_split")
    counts, displs = partition_counts(N, P)
    c = int(counts[rank])
    return codes[:c], flips[: max(c - 1, 0)], int(off.value)


def gray_general(n, q):
    N = q ** n
    xtab = np.zeros(max(N * n, 1), dtype=np.int64)
    flips = np.zeros(max(N - 1, 1), dtype=np.int64)
    _check(lib().or_gray_general(n, q, xtab.ctypes.data_as(_i64p), flips.ctypes.data_as(_i64p)), "gray_general")
    # column-major n x N (column k = code k), returned as (n, N) like the reference
    return xtab[: N * n].reshape(N, n).T.copy(), flips[: N - 1]


def partition_counts(n, P):
    c = np.zeros(P, dtype=np.int64)
    d = np.zeros(P, dtype=np.int64)
    lib().or_partition_counts(n, P, c.ctypes.data_as(_i64p), d.ctypes.data_as(_i64p))
    return c, d


def fwht(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.float64)).copy()
    L = int(np.log2(a.size))
    assert (1 << L) == a.size
    lib().or_fwht(a.ctypes.data_as(_dp), L)
    return a


def fht_qutrit(v):
    a, p = _cplx(np.asarray(v, dtype=np.complex128).copy())
    lib().or_fht_qutrit(p, a.size)
    return a


def sre_sums(psi, q, istart, iend, nthreads=None):
    """Raw (p2SAM, mSAM) over 1-based Gray indices [istart, iend]."""
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    p2, m = ctypes.c_double(), ctypes.c_double()
    _check(lib().or_sre_sums(p, n, float(q), istart, iend, nthreads or nthreads_default(), ctypes.byref(p2),
                             ctypes.byref(m)), "sre_sums")
    return p2.value, m.value


def sre_sums_fast(psi, qs, istart, iend, nthreads=None, per_thread=0):
    """Double-double sums over 1-based Gray indices [istart, iend], several q per
    transform: returns (p2 (hi, lo), m (nq, 2) as (hi, lo) rows).  per_thread > 0: each
    thread takes only the first per_thread indices of its slice (a timed sample)."""
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    q = np.ascontiguousarray(qs, dtype=np.float64).reshape(-1)
    out = np.zeros(2 * (1 + q.size))
    _check(lib().or_sre_sums_fast(p, n, q.ctypes.data_as(_dp), q.size, istart, iend, int(per_thread),
                                  nthreads or nthreads_default(), out.ctypes.data_as(_dp)), "sre_sums_fast")
    return out[:2].copy(), out[2:].reshape(q.size, 2).copy()


def sre(psi, q, nthreads=None):
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    assert (1 << n) == a.size
    s, l = ctypes.c_double(), ctypes.c_double()
    _check(lib().or_sre(p, n, float(q), nthreads or nthreads_default(), ctypes.byref(s), ctypes.byref(l)), "sre")
    return s.value, l.value


def naive_sre(psi, q, nthreads=None):
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    out = ctypes.c_double()
    _check(lib().or_naive_sre(p, n, int(q), nthreads or nthreads_default(), ctypes.byref(out)), "naive_sre")
    return out.value


def mc_sre_beta(psi, q, beta, prop_delta, rs):
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    pd = np.ascontiguousarray(prop_delta, dtype=np.uint64)
    r = np.ascontiguousarray(rs, dtype=np.float64)
    out = np.zeros(5)
    masks = np.zeros(pd.size, dtype=np.uint64)
    _check(lib().or_mc_sre_beta(p, n, float(q), pd.size, float(beta), pd.ctypes.data_as(_u64p),
                                r.ctypes.data_as(_dp), out.ctypes.data_as(_dp), masks.ctypes.data_as(_u64p)),
           "mc_sre_beta")
    return out, masks


def simpson_uniform(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().or_simpson_uniform(x.ctypes.data_as(_dp), y.ctypes.data_as(_dp), x.size)


def mc_sre(psi, q, nbeta, nsamples, prop_delta, rs, nthreads=None):
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    pd = np.ascontiguousarray(prop_delta, dtype=np.uint64).reshape(-1)
    r = np.ascontiguousarray(rs, dtype=np.float64).reshape(-1)
    assert pd.size == nbeta * nsamples and r.size == nbeta * nsamples
    M2, M2ADD, P2 = np.zeros(nbeta), np.zeros(nbeta), np.zeros(nbeta)
    m2 = ctypes.c_double()
    _check(lib().or_mc_sre(p, n, float(q), nbeta, nsamples, pd.ctypes.data_as(_u64p), r.ctypes.data_as(_dp),
                           nthreads or nthreads_default(), ctypes.byref(m2), M2.ctypes.data_as(_dp),
                           M2ADD.ctypes.data_as(_dp), P2.ctypes.data_as(_dp)), "mc_sre")
    return m2.value, M2, M2ADD, P2


def mana_sum(psi, istart, iend, nthreads=None):
    a, p = _cplx(psi)
    L = int(round(np.log(a.size) / np.log(3)))
    out = ctypes.c_double()
    _check(lib().or_mana_sum(p, L, istart, iend, nthreads or nthreads_default(), ctypes.byref(out)), "mana_sum")
    return out.value


def mana_pure(psi, nthreads=None):
    a, p = _cplx(psi)
    L = int(round(np.log(a.size) / np.log(3)))
    assert 3 ** L == a.size
    out = ctypes.c_double()
    _check(lib().or_mana_pure(p, L, nthreads or nthreads_default(), ctypes.byref(out)), "mana_pure")
    return out.value


def single_qutrit_M():
    out = np.zeros(81, dtype=np.complex128)
    lib().or_single_qutrit_M(out.view(np.float64).ctypes.data_as(_dp))
    return out.reshape(9, 9)


def mana_mixed(rho, return_w=False):
    """rho: (3^N, 3^N) complex matrix (numpy, any order); passed column-major."""
    r = np.asarray(rho, dtype=np.complex128)
    dim = r.shape[0]
    N = int(round(np.log(dim) / np.log(3)))
    assert 3 ** N == dim and r.shape == (dim, dim)
    col = np.ascontiguousarray(r.T)  # row-major of r.T == column-major of r
    w = np.zeros(9 ** N, dtype=np.complex128)
    out = ctypes.c_double()
    _check(lib().or_mana_mixed(col.view(np.float64).ctypes.data_as(_dp), N, ctypes.byref(out),
                               w.view(np.float64).ctypes.data_as(_dp)), "mana_mixed")
    return (out.value, w) if return_w else out.value


def sre_grad(psi, q=2, nthreads=None):
    a, p = _cplx(psi)
    n = int(np.log2(a.size))
    g = np.zeros(a.size, dtype=np.complex128)
    s = ctypes.c_double()
    _check(lib().or_sre_grad(p, n, float(q), nthreads or nthreads_default(), ctypes.byref(s),
                             g.view(np.float64).ctypes.data_as(_dp)), "sre_grad")
    return s.value, g  # g.real = dSRE/dRe psi, g.imag = dSRE/dIm psi


def _gate_buf(gate):
    g = np.asfortranarray(np.asarray(gate, dtype=np.complex128))
    return np.ascontiguousarray(g.T.reshape(-1))  # column-major element order


def apply_2gate(psi, q, gate, s1, s2):
    """src/State.jl:254-345: returns the state after the two-site gate (sites 1-based)."""
    a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128)).copy()
    n = int(round(np.log(a.size) / np.log(q)))
    g = _gate_buf(gate)
    _check(lib().or_apply_2gate(a.view(np.float64).ctypes.data_as(_dp), n, q,
                                g.view(np.float64).ctypes.data_as(_dp), s1, s2), "or_apply_2gate")
    return a


def brick_wall(psi, q, depth, gates):
    """src/State.jl:200-221 with the given layer-order gate list."""
    a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128)).copy()
    n = int(round(np.log(a.size) / np.log(q)))
    gs = np.ascontiguousarray(np.concatenate([_gate_buf(g) for g in gates])) if len(gates) else np.zeros(1, complex)
    _check(lib().or_brick_wall(a.view(np.float64).ctypes.data_as(_dp), n, q, depth,
                               gs.view(np.float64).ctypes.data_as(_dp), len(gates)), "or_brick_wall")
    return a


def reduced_density_matrix(psi, q, NA, side="right"):
    """src/DensityMatrix.jl:94-123; returns the dimA x dimA matrix."""
    a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128))
    n = int(round(np.log(a.size) / np.log(q)))
    dimA = q ** NA
    rho = np.zeros(dimA * dimA, dtype=np.complex128)
    _check(lib().or_reduced_density_matrix(a.view(np.float64).ctypes.data_as(_dp), n, q, NA,
                                           0 if side == "left" else 1, rho.view(np.float64).ctypes.data_as(_dp)),
           "or_reduced_density_matrix")
    return rho.reshape(dimA, dimA, order="F")
