"""ctypes binding of libhadamag_b200.so (declared in include/hadamag_b200.h).

The library is the only compute path: nothing here computes an SRE or Mana value on
the CPU.  If the shared object is missing or no CUDA device is visible, every call
raises instead of falling back.
"""
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhadamag_b200.so")

HM_OK = 0
HM_ERR_ARG = -1
HM_ERR_SIZE = -2
HM_ERR_Q = -3
HM_ERR_CUDA = -4
HM_ERR_OOM = -5
HM_ERR_TIMEOUT = -6
HM_ERR_ALIGN = -7

HM_FP64 = 0
HM_FP32 = 1
HM_PLAIN = 2
PRECISIONS = {"fp64": HM_FP64, "fp32": HM_FP32, "plain": HM_PLAIN}

# every entry point declared in include/hadamag_b200.h
EXPORTS = [
    "hm_abi_version", "hm_create", "hm_destroy", "hm_last_error", "hm_set_stream", "hm_last_kernel_ms",
    "hm_sre", "hm_sre_dev", "hm_sre_range", "hm_sre_range_dev", "hm_sre_batched", "hm_sre_grad",
    "hm_mc_sre", "hm_mana_pure", "hm_mana_mixed", "hm_gray_table", "hm_gray_table_general", "hm_set_param",
    "hm_last_launch_count", "hm_probe_fp64_peak", "hm_probe_fp32_peak", "hm_sre_noalloc", "hm_autotune",
    "hm_apply_2gate", "hm_brick_wall", "hm_reduced_density_matrix", "hm_mc_sre_chains", "hm_mana_pure_range",
    "hm_sre_multi", "hm_sre_range_multi", "hm_multi_last_error", "hm_multi_release",
    "hm_load_state", "hm_free_state", "hm_io_last_error", "hm_gray_table_split", "hm_autotune_choice",
]
HM_PARAM_BATCH = 1
HM_PARAM_RING = 2
HM_PARAM_UNITS = 3
HM_PARAM_GRAPH = 4
HM_PARAM_ADJ_BATCH = 5
HM_PARAM_ENGINE = 6
HM_PARAM_QUEUE_SLOTS = 7
HM_PARAM_QUEUE_SLOT_MIB = 8
HM_PARAM_QUEUE_CHUNK = 9
HM_PARAM_QUEUE_CTAS = 10
HM_PARAM_QUEUE_STALL_TEST = 11
HM_PARAM_QUEUE_LEAD = 12
HM_PARAM_BATCH_SPLIT_N = 14


class ArgumentError(ValueError):
    """Invalid argument (the reference raises Julia's ArgumentError in the same places)."""


class HadaMAGError(RuntimeError):
    """A CUDA or device-side failure reported by libhadamag_b200.so."""


_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

_lib = None
_lib_lock = threading.Lock()


def load_library(path=None):
    """Load (once) and return the CDLL with argument types declared."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise HadaMAGError(
                f"{p} is missing: build it with `python hadamag.jl_b200/build.py` (there is no CPU fallback)")
        L = ctypes.CDLL(p)
        i, d, u64 = ctypes.c_int, ctypes.c_double, ctypes.c_uint64
        L.hm_abi_version.restype = i
        L.hm_create.argtypes = [ctypes.POINTER(_vp), i]
        L.hm_destroy.argtypes = [_vp]
        L.hm_last_error.argtypes = [_vp]
        L.hm_last_error.restype = ctypes.c_char_p
        L.hm_set_stream.argtypes = [_vp, _vp]
        L.hm_last_kernel_ms.argtypes = [_vp, _dp]
        L.hm_sre.argtypes = [_vp, _dp, i, _dp, i, i, _dp, _dp]
        L.hm_sre_dev.argtypes = [_vp, _vp, i, _dp, i, i, _dp, _dp]
        L.hm_sre_range.argtypes = [_vp, _dp, i, u64, u64, _dp, i, i, _dp, _dp]
        L.hm_sre_range_dev.argtypes = [_vp, _vp, i, u64, u64, _dp, i, i, _dp, _dp]
        L.hm_sre_batched.argtypes = [_vp, i, ctypes.POINTER(_dp), _ip, _dp, i, i, _dp, _dp]
        L.hm_sre_grad.argtypes = [_vp, _dp, i, d, _dp, _dp]
        L.hm_mc_sre.argtypes = [_vp, _dp, i, d, i, i, _u64p, _dp, _dp, _dp, _dp, _dp, _u64p]
        L.hm_mana_pure.argtypes = [_vp, _dp, i, _dp]
        L.hm_mana_mixed.argtypes = [_vp, _dp, i, _dp]
        L.hm_gray_table.argtypes = [_vp, i, _u64p, _i64p]
        L.hm_gray_table_general.argtypes = [_vp, i, i, _i64p, _i64p]
        L.hm_set_param.argtypes = [i, i]
        L.hm_last_launch_count.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
        L.hm_probe_fp64_peak.argtypes = [_vp, _dp]
        L.hm_probe_fp32_peak.argtypes = [_vp, _dp]
        L.hm_sre_noalloc.argtypes = [_dp, i, _dp, i, _dp, _dp, _vp]
        L.hm_autotune.argtypes = [_vp, i, i, _ip, _dp]
        L.hm_mc_sre_chains.argtypes = [_vp, _dp, i, d, i, i, i, i, _u64p, _dp, _dp, _dp, _dp, _u64p]
        L.hm_mana_pure_range.argtypes = [_vp, _dp, i, ctypes.c_int64, ctypes.c_int64, _dp]
        L.hm_apply_2gate.argtypes = [_vp, _dp, i, i, _dp, i, i]
        L.hm_brick_wall.argtypes = [_vp, _dp, i, i, i, _dp, i]
        L.hm_reduced_density_matrix.argtypes = [_vp, _dp, i, i, i, i, _dp]
        L.hm_sre_multi.argtypes = [_ip, i, _dp, i, _dp, i, i, _dp, _dp]
        L.hm_sre_range_multi.argtypes = [_ip, i, _dp, i, ctypes.c_uint64, ctypes.c_uint64, _dp, i, i, _dp, _dp]
        L.hm_multi_last_error.argtypes = []
        L.hm_multi_last_error.restype = ctypes.c_char_p
        L.hm_multi_release.argtypes = []
        L.hm_autotune_choice.argtypes = [i, i, _ip, _ip, _ip]
        L.hm_gray_table_split.argtypes = [_vp, i, i, i, i, _i64p, _i64p, _i64p, _i64p]
        L.hm_load_state.argtypes = [ctypes.c_char_p, i, ctypes.POINTER(_dp), ctypes.POINTER(ctypes.c_uint64)]
        L.hm_free_state.argtypes = [_dp]
        L.hm_io_last_error.argtypes = []
        L.hm_io_last_error.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name not in ("hm_last_error", "hm_abi_version", "hm_multi_last_error", "hm_io_last_error"):
                getattr(L, name).restype = i
        _lib = L
        return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _cplx(psi):
    a = np.ascontiguousarray(np.asarray(psi), dtype=np.complex128)
    return a, a.view(np.float64).ctypes.data_as(_dp)


class Context:
    """One CUDA device, one stream and the device buffers of libhadamag_b200.so."""

    def __init__(self, device=0):
        self.lib = load_library()
        h = _vp()
        rc = self.lib.hm_create(ctypes.byref(h), int(device))
        if rc != HM_OK:
            raise HadaMAGError(f"hm_create(device={device}) failed with status {rc} (no usable CUDA device?)")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.hm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc == HM_OK:
            return
        msg = self.lib.hm_last_error(self.handle).decode(errors="replace")
        if rc in (HM_ERR_ARG, HM_ERR_SIZE, HM_ERR_Q, HM_ERR_ALIGN):
            raise ArgumentError(f"{what}: {msg}")
        raise HadaMAGError(f"{what} failed with status {rc}: {msg}")

    def set_stream(self, stream_handle):
        self._check(self.lib.hm_set_stream(self.handle, _vp(stream_handle or 0)), "hm_set_stream")

    def last_launch_count(self):
        v = ctypes.c_longlong()
        self._check(self.lib.hm_last_launch_count(self.handle, ctypes.byref(v)), "hm_last_launch_count")
        return v.value

    def probe_fp64_peak(self):
        v = ctypes.c_double()
        self._check(self.lib.hm_probe_fp64_peak(self.handle, ctypes.byref(v)), "hm_probe_fp64_peak")
        return v.value

    def probe_fp32_peak(self):
        v = ctypes.c_double()
        self._check(self.lib.hm_probe_fp32_peak(self.handle, ctypes.byref(v)), "hm_probe_fp32_peak")
        return v.value

    def autotune(self, n, precision=HM_FP64):
        """Pick and record the two-pass batch size for (n, precision); returns
        (X, microseconds per X-string)."""
        x = ctypes.c_int()
        us = ctypes.c_double()
        self._check(self.lib.hm_autotune(self.handle, int(n), int(precision), ctypes.byref(x), ctypes.byref(us)),
                    "hm_autotune")
        return x.value, us.value

    def last_kernel_ms(self):
        v = ctypes.c_double()
        self._check(self.lib.hm_last_kernel_ms(self.handle, ctypes.byref(v)), "hm_last_kernel_ms")
        return v.value

    # ------------------------------------------------------------------ exact SRE
    def sre(self, psi, qs=(2.0,), precision=HM_FP64):
        a, p = _cplx(psi)
        n = _log2_exact(a.size)
        q = _f64(qs)
        out = np.zeros(q.size)
        lost = ctypes.c_double()
        self._check(self.lib.hm_sre(self.handle, p, n, q.ctypes.data_as(_dp), q.size, int(precision),
                                    out.ctypes.data_as(_dp), ctypes.byref(lost)), "hm_sre")
        return out, lost.value

    def sre_dev(self, psi_dev_ptr, n, qs=(2.0,), precision=HM_FP64):
        q = _f64(qs)
        out = np.zeros(q.size)
        lost = ctypes.c_double()
        self._check(self.lib.hm_sre_dev(self.handle, _vp(psi_dev_ptr), int(n), q.ctypes.data_as(_dp), q.size,
                                        int(precision), out.ctypes.data_as(_dp), ctypes.byref(lost)), "hm_sre_dev")
        return out, lost.value

    def sre_range(self, psi, k_begin, k_end, qs=(2.0,), precision=HM_FP64):
        a, p = _cplx(psi)
        n = _log2_exact(a.size)
        q = _f64(qs)
        p2 = np.zeros(2)
        m = np.zeros(2 * q.size)
        self._check(self.lib.hm_sre_range(self.handle, p, n, int(k_begin), int(k_end), q.ctypes.data_as(_dp), q.size,
                                          int(precision), p2.ctypes.data_as(_dp), m.ctypes.data_as(_dp)),
                    "hm_sre_range")
        return p2, m.reshape(q.size, 2)

    def sre_range_dev(self, psi_dev_ptr, n, k_begin, k_end, qs=(2.0,), precision=HM_FP64):
        q = _f64(qs)
        p2 = np.zeros(2)
        m = np.zeros(2 * q.size)
        self._check(self.lib.hm_sre_range_dev(self.handle, _vp(psi_dev_ptr), int(n), int(k_begin), int(k_end),
                                              q.ctypes.data_as(_dp), q.size, int(precision),
                                              p2.ctypes.data_as(_dp), m.ctypes.data_as(_dp)), "hm_sre_range_dev")
        return p2, m.reshape(q.size, 2)

    def sre_batched(self, psis, qs=(2.0,), precision=HM_FP64):
        arrs = [np.ascontiguousarray(np.asarray(p), dtype=np.complex128) for p in psis]
        ns = np.array([_log2_exact(a.size) for a in arrs], dtype=np.int32)
        ptrs = (_dp * len(arrs))(*[a.view(np.float64).ctypes.data_as(_dp) for a in arrs])
        q = _f64(qs)
        out = np.zeros(len(arrs) * q.size)
        lost = np.zeros(len(arrs))
        self._check(self.lib.hm_sre_batched(self.handle, len(arrs), ptrs, ns.ctypes.data_as(_ip),
                                            q.ctypes.data_as(_dp), q.size, int(precision), out.ctypes.data_as(_dp),
                                            lost.ctypes.data_as(_dp)), "hm_sre_batched")
        return out.reshape(len(arrs), q.size), lost

    def sre_grad(self, psi, q=2.0):
        a, p = _cplx(psi)
        n = _log2_exact(a.size)
        g = np.zeros(a.size, dtype=np.complex128)
        v = ctypes.c_double()
        self._check(self.lib.hm_sre_grad(self.handle, p, n, float(q), ctypes.byref(v),
                                         g.view(np.float64).ctypes.data_as(_dp)), "hm_sre_grad")
        return v.value, g

    # ------------------------------------------------------------------ MC_SRE
    def mc_sre(self, psi, q, nbeta, nsamples, prop_delta, rs):
        a, p = _cplx(psi)
        n = _log2_exact(a.size)
        pd = np.ascontiguousarray(prop_delta, dtype=np.uint64).reshape(-1)
        r = _f64(rs).reshape(-1)
        if pd.size != nbeta * nsamples or r.size != nbeta * nsamples:
            raise ArgumentError("proposal stream must hold nbeta * nsamples entries")
        M2, M2ADD, P2 = np.zeros(nbeta), np.zeros(nbeta), np.zeros(nbeta)
        fm = np.zeros(nbeta, dtype=np.uint64)
        m2 = ctypes.c_double()
        self._check(self.lib.hm_mc_sre(self.handle, p, n, float(q), int(nbeta), int(nsamples),
                                       pd.ctypes.data_as(_u64p), r.ctypes.data_as(_dp), ctypes.byref(m2),
                                       M2.ctypes.data_as(_dp), M2ADD.ctypes.data_as(_dp), P2.ctypes.data_as(_dp),
                                       fm.ctypes.data_as(_u64p)), "hm_mc_sre")
        return m2.value, M2, M2ADD, P2, fm

    def mc_sre_chains(self, psi, q, nbeta, chain_begin, chain_end, nsamples, prop_delta, rs):
        """Chains [chain_begin, chain_end) of the nbeta-point beta grid; prop_delta / rs hold
        those chains' streams.  Returns (M2, M2ADD, P2, final_mask) per chain."""
        a, p = _cplx(psi)
        n = _log2_exact(a.size)
        nch = int(chain_end) - int(chain_begin)
        pd = np.ascontiguousarray(prop_delta, dtype=np.uint64).reshape(-1)
        r = _f64(rs).reshape(-1)
        if nch < 1 or pd.size != nch * nsamples or r.size != nch * nsamples:
            raise ArgumentError("proposal stream must hold (chain_end - chain_begin) * nsamples entries")
        M2, M2ADD, P2 = np.zeros(nch), np.zeros(nch), np.zeros(nch)
        fm = np.zeros(nch, dtype=np.uint64)
        self._check(self.lib.hm_mc_sre_chains(self.handle, p, n, float(q), int(nbeta), int(chain_begin),
                                              int(chain_end), int(nsamples), pd.ctypes.data_as(_u64p),
                                              r.ctypes.data_as(_dp), M2.ctypes.data_as(_dp),
                                              M2ADD.ctypes.data_as(_dp), P2.ctypes.data_as(_dp),
                                              fm.ctypes.data_as(_u64p)), "hm_mc_sre_chains")
        return M2, M2ADD, P2, fm

    # ------------------------------------------------------------------ Mana
    def mana_pure_range(self, psi, x_begin, x_end):
        """Double-double sum of |W| over the X-strings [x_begin, x_end) (natural order)."""
        a, p = _cplx(psi)
        L = _log3_exact(a.size)
        out = np.zeros(2)
        self._check(self.lib.hm_mana_pure_range(self.handle, p, L, int(x_begin), int(x_end),
                                                out.ctypes.data_as(_dp)), "hm_mana_pure_range")
        return out

    def mana_pure(self, psi):
        a, p = _cplx(psi)
        L = _log3_exact(a.size)
        v = ctypes.c_double()
        self._check(self.lib.hm_mana_pure(self.handle, p, L, ctypes.byref(v)), "hm_mana_pure")
        return v.value

    def mana_mixed(self, rho):
        r = np.asarray(rho, dtype=np.complex128)
        if r.ndim != 2 or r.shape[0] != r.shape[1]:
            raise ArgumentError("DensityMatrix must be square")
        N = _log3_exact(r.shape[0])
        col = np.ascontiguousarray(r.T)  # row-major bytes of r.T = column-major r
        v = ctypes.c_double()
        self._check(self.lib.hm_mana_mixed(self.handle, col.view(np.float64).ctypes.data_as(_dp), N,
                                           ctypes.byref(v)), "hm_mana_mixed")
        return v.value

    # ------------------------------------------------------------------ Gray tables
    def gray_table(self, n):
        N = 1 << n
        codes = np.zeros(N, dtype=np.uint64)
        flips = np.zeros(max(N - 1, 1), dtype=np.int64)
        self._check(self.lib.hm_gray_table(self.handle, int(n), codes.ctypes.data_as(_u64p),
                                           flips.ctypes.data_as(_i64p)), "hm_gray_table")
        return codes, flips[: N - 1]

    def gray_table_split(self, n, q, rank, P):
        """Rank's slice of the Gray table split over P processes (hm_gray_table_split):
        q = 2 -> (codes uint64[cnt], flips, code_off); q > 2 -> (XTAB (n, cnt), flips, code_off)."""
        N = q ** n
        cap = -(-N // P)
        width = 1 if q == 2 else n
        codes = np.zeros(max(cap * width, 1), dtype=np.int64)
        flips = np.zeros(max(cap, 1), dtype=np.int64)
        off, cnt = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.hm_gray_table_split(self.handle, int(n), int(q), int(rank), int(P),
                                                 codes.ctypes.data_as(_i64p), flips.ctypes.data_as(_i64p),
                                                 ctypes.byref(off), ctypes.byref(cnt)), "hm_gray_table_split")
        c = cnt.value
        fl = flips[: max(c - 1, 0)]
        if q == 2:
            return codes[:c].view(np.uint64), fl, off.value
        return codes[: c * n].reshape(c, n).T.copy(), fl, off.value

    def apply_2gate(self, psi, q, gate, s1, s2):
        """Two-site gate on sites s1, s2 (1-based); returns the new amplitudes."""
        a = np.array(psi, dtype=np.complex128, copy=True)
        n = _logq_exact(a.size, q)
        g = _gate_colmajor(gate, q)
        self._check(self.lib.hm_apply_2gate(self.handle, a.view(np.float64).ctypes.data_as(_dp), n, int(q),
                                            g.view(np.float64).ctypes.data_as(_dp), int(s1), int(s2)),
                    "hm_apply_2gate")
        return a

    def brick_wall(self, psi, q, depth, gates):
        """Brick-wall circuit with one gate per site pair, in layer order."""
        a = np.array(psi, dtype=np.complex128, copy=True)
        n = _logq_exact(a.size, q)
        gs = (np.ascontiguousarray(np.concatenate([_gate_colmajor(g, q) for g in gates])) if len(gates)
              else np.zeros(1, dtype=np.complex128))
        self._check(self.lib.hm_brick_wall(self.handle, a.view(np.float64).ctypes.data_as(_dp), n, int(q),
                                           int(depth), gs.view(np.float64).ctypes.data_as(_dp), len(gates)),
                    "hm_brick_wall")
        return a

    def reduced_density_matrix(self, psi, q, NA, side="right"):
        """rho_A (q^NA x q^NA) of the NA least ("left") or most ("right") significant sites."""
        a = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128))
        n = _logq_exact(a.size, q)
        if side not in ("left", "right"):
            raise ArgumentError(f"side must be :left or :right (got {side})")
        if not 0 <= NA <= n:
            raise ArgumentError(f"need 0 ≤ NA ≤ N (got NA={NA}, N={n})")
        dimA = q ** NA
        rho = np.zeros(dimA * dimA, dtype=np.complex128)
        self._check(self.lib.hm_reduced_density_matrix(self.handle, a.view(np.float64).ctypes.data_as(_dp), n,
                                                       int(q), int(NA), 0 if side == "left" else 1,
                                                       rho.view(np.float64).ctypes.data_as(_dp)),
                    "hm_reduced_density_matrix")
        return rho.reshape(dimA, dimA, order="F")

    def gray_table_general(self, n, q):
        N = q ** n
        xt = np.zeros(max(N * n, 1), dtype=np.int64)
        flips = np.zeros(max(N - 1, 1), dtype=np.int64)
        self._check(self.lib.hm_gray_table_general(self.handle, int(n), int(q), xt.ctypes.data_as(_i64p),
                                                   flips.ctypes.data_as(_i64p)), "hm_gray_table_general")
        return xt[: N * n].reshape(N, n).T.copy(), flips[: N - 1]


def _logq_exact(size, q):
    if q not in (2, 3):
        raise ArgumentError(f"only q=2 and q=3 are implemented (got q={q})")
    n, t = 0, 1
    while t < size:
        t *= q
        n += 1
    if t != size:
        raise ArgumentError(f"length(psi)={size} is not a power of q={q}")
    return n


def _gate_colmajor(gate, q):
    g = np.asarray(gate, dtype=np.complex128)
    if g.shape != (q * q, q * q):
        raise ArgumentError(f"gate must be of size (q^2 × q^2) = ({q * q}, {q * q}), got {g.shape}")
    return np.ascontiguousarray(g.T).reshape(-1)  # column-major element order


def _log2_exact(size):
    n = int(size).bit_length() - 1
    if size < 1 or (1 << n) != size:
        raise ArgumentError(f"length(vec)={size} is not a power of q=2")
    return n


def _log3_exact(size):
    n, t = 0, int(size)
    while t % 3 == 0 and t > 1:
        t //= 3
        n += 1
    if t != 1:
        raise ArgumentError(f"length(vec)={size} is not a power of q=3")
    return n


def _multi_check(rc, what):
    if rc == HM_OK:
        return
    msg = load_library().hm_multi_last_error().decode(errors="replace")
    if rc in (HM_ERR_ARG, HM_ERR_SIZE, HM_ERR_Q, HM_ERR_ALIGN):
        raise ArgumentError(f"{what}: {msg}")
    raise HadaMAGError(f"{what} failed with status {rc}: {msg}")


def sre_multi(devices, psi, qs=(2.0,), precision=HM_FP64):
    """Exact SRE over several GPUs in one call (hm_sre_multi); returns (values, lost_norm)."""
    L = load_library()
    a, p = _cplx(psi)
    n = _log2_exact(a.size)
    d = np.ascontiguousarray(devices, dtype=np.int32)
    q = _f64(qs)
    out = np.zeros(q.size)
    lost = ctypes.c_double()
    _multi_check(L.hm_sre_multi(d.ctypes.data_as(_ip), d.size, p, n, q.ctypes.data_as(_dp), q.size, int(precision),
                                out.ctypes.data_as(_dp), ctypes.byref(lost)), "hm_sre_multi")
    return out, lost.value


def sre_range_multi(devices, psi, k_begin, k_end, qs=(2.0,), precision=HM_FP64):
    """Double-double sums of the Gray range [k_begin, k_end) split over several GPUs."""
    L = load_library()
    a, p = _cplx(psi)
    n = _log2_exact(a.size)
    d = np.ascontiguousarray(devices, dtype=np.int32)
    q = _f64(qs)
    p2 = np.zeros(2)
    m = np.zeros(2 * q.size)
    _multi_check(L.hm_sre_range_multi(d.ctypes.data_as(_ip), d.size, p, n, int(k_begin), int(k_end),
                                      q.ctypes.data_as(_dp), q.size, int(precision), p2.ctypes.data_as(_dp),
                                      m.ctypes.data_as(_dp)), "hm_sre_range_multi")
    return p2, m.reshape(q.size, 2)


def load_state_pinned(path, q=2):
    """hm_load_state: the file's amplitudes in page-locked host memory, as a complex128
    numpy array that frees the buffer when it is garbage-collected."""
    import weakref
    L = load_library()
    ptr = _dp()
    n = ctypes.c_uint64()
    rc = L.hm_load_state(str(path).encode(), int(q), ctypes.byref(ptr), ctypes.byref(n))
    if rc != HM_OK:
        msg = L.hm_io_last_error().decode(errors="replace")
        raise (ArgumentError if rc in (HM_ERR_ARG, HM_ERR_SIZE) else HadaMAGError)(msg)
    buf = (ctypes.c_double * (2 * n.value)).from_address(ctypes.addressof(ptr.contents))
    weakref.finalize(buf, L.hm_free_state, ptr)
    return np.frombuffer(buf, dtype=np.complex128)


def multi_release():
    load_library().hm_multi_release()


def autotune_choice(n, precision=HM_FP64):
    """(engine, batch, CTAs per SM) that hm_autotune recorded for (n, precision); engine
    0 = not tuned, 1 = stage kernels, 2 = queue sweep."""
    e, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = load_library().hm_autotune_choice(int(n), int(precision), ctypes.byref(e), ctypes.byref(b), ctypes.byref(c))
    if rc != HM_OK:
        raise ArgumentError(f"hm_autotune_choice({n}, {precision}) rejected")
    return e.value, b.value, c.value


def set_param(param, value):
    """Process-wide tuning knob (HM_PARAM_BATCH, _RING, _UNITS, _GRAPH, _ADJ_BATCH, _ENGINE, _QUEUE_SLOTS,
    _QUEUE_SLOT_MIB, _QUEUE_CHUNK, _QUEUE_CTAS); 0 restores the default."""
    rc = load_library().hm_set_param(int(param), int(value))
    if rc != HM_OK:
        raise ArgumentError(f"hm_set_param({param}, {value}) rejected")


_default_ctx = {}


def default_context(device=0):
    """Process-wide context per device (created on first use)."""
    ctx = _default_ctx.get(device)
    if ctx is None or ctx.handle is None:
        ctx = Context(device)
        _default_ctx[device] = ctx
    return ctx
