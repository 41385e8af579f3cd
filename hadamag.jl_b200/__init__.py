"""hadamag_b200 -- HadaMAG.jl's exact-SRE / MC_SRE / Mana hot path on NVIDIA B200.

Python mirror of the reference's user API (src/HadaMAG.jl:1-25): the same names,
argument meanings and error behaviour, served by one backend, ``:b200``, which calls
libhadamag_b200.so (hand-written sm_100a kernels behind a C ABI, see
include/hadamag_b200.h).  There is no CPU fallback: without the shared object or a
CUDA device every compute call raises.

    import hadamag_b200 as hm
    psi = hm.StateVec(vec)              # vec: complex128, length 2^n
    value, lost_norm = hm.SRE(psi, 2)   # src/SRE.jl:75-83
    m2 = hm.MC_SRE(psi, 2, Nbeta=13, Nsamples=1000, seed=123)
    mana = hm.Mana(hm.StateVec(v3, q=3))          # src/Mana.jl:15-17
    mana_rho = hm.Mana(hm.DensityMatrix(rho, q=3))  # src/Mana.jl:305-314

The package directory is ``hadamag.jl_b200/``; the repository root's
``hadamag_b200.py`` makes it importable as ``hadamag_b200``.
"""
import os
import warnings

import numpy as np

from . import _native  # noqa: F401
from . import shard  # noqa: F401  (multi-GPU Gray-range split)
from ._native import (HM_FP32, HM_FP64, HM_PLAIN, PRECISIONS, ArgumentError, Context, HadaMAGError,
                      default_context, load_library)

__all__ = [
    "StateVec", "DensityMatrix", "SRE", "MC_SRE", "Mana", "SRE_batched", "SRE_grad", "generate_gray_table",
    "load_state", "reduced_density_matrix", "proposal_stream", "qubits", "qudits", "qudit_dim", "data",
    "haar_random_unitary", "brick_wall_pairs", "apply_2gate", "apply_2gate_inplace", "apply_brick_wall",
    "apply_brick_wall_haar", "rand_haar", "rand_cliff",
    "ArgumentError", "HadaMAGError", "Context", "B200",
]


# ----------------------------------------------------------------------------------
# containers (src/State.jl:11-63, src/DensityMatrix.jl:8-41)

def _power_q(length, q):
    """(n, is_power) with length == q^n, as _power_q of src/Helpers.jl:7-15."""
    n, tmp = 0, int(length)
    while tmp > 0 and tmp % q == 0:
        tmp //= q
        n += 1
    return n, tmp == 1


class StateVec:
    """Pure state of n q-dits; ``data`` is a complex128 vector of length q^n.

    Raises ArgumentError when the length is not a power of q (src/State.jl:40-44).
    """

    def __init__(self, vec, q=2, copy=True):
        v = (np.array(vec, dtype=np.complex128) if copy else np.asarray(vec, dtype=np.complex128)).reshape(-1)
        n, ok = _power_q(v.size, q)
        if not ok:
            raise ArgumentError(f"length(vec)={v.size} is not a power of q={q}")
        self.data, self.n, self.q = v, n, q

    def __len__(self):
        return self.data.size

    def __repr__(self):
        return f"StateVec{{ComplexF64,{self.q}}}(n={self.n}, dim={self.data.size})"

    def normalize(self):
        self.data /= np.linalg.norm(self.data)
        return self


class DensityMatrix:
    """Mixed state of n q-dits; ``data`` is a complex128 q^n x q^n matrix.

    Raises ArgumentError when the matrix is not square or its size is not a power of q
    (src/DensityMatrix.jl:28-35).
    """

    def __init__(self, mat, q=2):
        m = np.array(mat, dtype=np.complex128)
        if m.ndim != 2 or m.shape[0] != m.shape[1]:
            raise ArgumentError("DensityMatrix must be square")
        n, ok = _power_q(m.shape[0], q)
        if not ok:
            raise ArgumentError(f"size(mat,1)={m.shape[0]} is not a power of q={q}")
        self.data, self.n, self.q = m, n, q

    def __repr__(self):
        return f"DensityMatrix{{ComplexF64,{self.q}}}(n={self.n}, size={self.data.shape})"


def qudits(s):
    return s.n


def qubits(s):
    if s.q != 2:
        raise ArgumentError("qubits() is defined for q = 2 states")
    return s.n


def qudit_dim(s):
    return s.q


def data(s):
    return s.data


# ----------------------------------------------------------------------------------
# backend selection (src/Backends/Dispatch.jl:4-90)

class B200:
    """The sm_100a backend.  ``device`` selects the CUDA device; ``devices`` (a list) runs
    the exact SRE over several GPUs in one call, each sweeping a contiguous share of the
    Gray range (the :mpi_cuda backend's per-node split, ext/HadaMAGMPICUDAExt.jl:49-95)."""

    def __init__(self, device=0, devices=None):
        self.devices = list(devices) if devices else None
        self.device = self.devices[0] if self.devices else device

    def context(self):
        return default_context(self.device)


def _choose_backend(b, device=0):
    """``:b200`` (or ``:auto`` / None, since it is the only backend of this package).

    The reference's CPU, MPI and CUDA.jl backends live in HadaMAG.jl itself; asking this
    package for them is an ArgumentError rather than a silent substitution.
    """
    if isinstance(b, B200):
        return b
    name = (b or "auto").lstrip(":") if isinstance(b, str) or b is None else str(b)
    if name in ("b200", "auto"):
        return B200(device)
    raise ArgumentError(f"backend :{name} is provided by HadaMAG.jl; this package implements :b200")


def _progress_warning(progress):
    if progress:
        warnings.warn("Progress bar not implemented for the b200 backend.", stacklevel=3)


def _precision(p):
    if isinstance(p, int):
        return p
    try:
        return PRECISIONS[str(p).lower()]
    except KeyError:
        raise ArgumentError(f"precision must be one of {sorted(PRECISIONS)} (got {p!r})") from None


def _as_state(psi, q):
    if isinstance(psi, StateVec):
        if psi.q != q:
            raise ArgumentError(f"expected a StateVec with q={q}, got q={psi.q}")
        return psi
    return StateVec(psi, q=q)


# ----------------------------------------------------------------------------------
# user API

def SRE(psi, q, backend="auto", progress=False, precision="fp64", device=0):
    """Exact stabilizer Renyi entropy; returns (value, lost_norm).

    value = -log2(sum_P <psi|P|psi>^(2q) / 2^n) over all 4^n Pauli strings and
    lost_norm = |1 - sum_P <psi|P|psi>^2 / 2^n|, as src/SRE.jl:75-83 and
    src/Backends/Threads.jl:108-159 (for q != 2 the value is (q-1) M_q, as there).
    precision: "fp64" (default), "fp32" (FP32 butterflies, FP64 reductions) or "plain"
    (the reference CUDA backend's multi-launch structure, FP64).
    """
    _progress_warning(progress)
    be = _choose_backend(backend, device)
    s = _as_state(psi, 2)
    if be.devices and len(be.devices) > 1:
        vals, lost = _native.sre_multi(be.devices, s.data, (float(q),), _precision(precision))
    else:
        vals, lost = be.context().sre(s.data, (float(q),), _precision(precision))
    return float(vals[0]), float(lost)


def SRE_batched(psis, qs=(2,), precision="fp64", device=0):
    """Exact SRE of many states (qubit counts may differ) in one launch sequence.

    Returns (values[nstates, len(qs)], lost_norm[nstates]).  No reference counterpart.
    """
    states = [_as_state(p, 2).data for p in psis]
    return default_context(device).sre_batched(states, tuple(float(q) for q in qs), _precision(precision))


def SRE_grad(psi, q=2, device=0):
    """Value and gradient of the exact SRE_q; grad.real = dSRE/dRe(psi), grad.imag =
    dSRE/dIm(psi).  No reference counterpart (hand-written adjoint kernel)."""
    s = _as_state(psi, 2)
    return default_context(device).sre_grad(s.data, float(q))


def proposal_stream(L, Nbeta, Nsamples, seed=None):
    """Metropolis proposal stream with the distribution of src/SRE.jl:142-170.

    Chain i (1-based) uses seed + i: tries[t] = floor(9 u) + 1 single-site flips with
    sites uniform in 1..L, XOR-ed into prop_delta[t]; rs[t] uniform in [0, 1).  Julia's
    MersenneTwister stream itself cannot be regenerated outside Julia; the Julia
    backend passes the reference's own draws through the same C ABI.
    """
    base = int(np.random.default_rng().integers(1, 10**9)) if seed is None else int(seed)
    pd = np.zeros((Nbeta, Nsamples), dtype=np.uint64)
    rs = np.zeros((Nbeta, Nsamples), dtype=np.float64)
    for i in range(Nbeta):
        g = np.random.default_rng(base + i + 1)
        u = g.random(Nsamples)
        tries = np.floor(u * 9).astype(np.int64) + 1
        rs[i] = g.random(Nsamples)
        sites = g.integers(0, L, size=int(tries.sum()))
        bits = (np.uint64(1) << sites.astype(np.uint64))
        idx = np.repeat(np.arange(Nsamples), tries)
        np.bitwise_xor.at(pd[i], idx, bits)
    return pd, rs


def MC_SRE(psi, q, backend="auto", Nbeta=13, Nsamples=1000, seed=None, progress=False, device=0,
           prop_delta=None, rs=None):
    """Monte-Carlo SRE_q (src/SRE.jl:33-43, src/Backends/Threads.jl:161-221).

    Nbeta chains at beta_i = (i-1)/(Nbeta-1) (Nbeta odd, Simpson's rule); returns
    -log2(2^-I + I_add).  The proposal stream comes from proposal_stream(seed) unless
    given explicitly (prop_delta, rs with shape (Nbeta, Nsamples)).
    """
    _progress_warning(progress)
    if Nbeta % 2 != 1:
        raise ArgumentError("Simpson needs an odd number of β points.")
    be = _choose_backend(backend, device)
    s = _as_state(psi, 2)
    if prop_delta is None or rs is None:
        prop_delta, rs = proposal_stream(s.n, Nbeta, Nsamples, seed)
    m2, _, _, _, _ = be.context().mc_sre(s.data, float(q), Nbeta, Nsamples, prop_delta, rs)
    return m2


def Mana(psi, backend="auto", progress=False, device=0):
    """Mana of a qutrit state.

    StateVec (q=3): log2(sum |W|) / log2(3) over the phase-space transforms of every
    ternary X-string (src/Mana.jl:15-92, src/Backends/Threads.jl:223-271).
    DensityMatrix (q=3): log2(sum |M^(x)N vec9(rho)| / 3^N) (src/Mana.jl:305-314).
    """
    _progress_warning(progress)
    if isinstance(psi, DensityMatrix):
        if psi.q != 3:
            raise ArgumentError("Mana needs a qutrit DensityMatrix (q=3)")
        return default_context(device).mana_mixed(psi.data)
    be = _choose_backend(backend, device)
    s = _as_state(psi, 3)
    return be.context().mana_pure(s.data)


def autotune(n, precision="fp64", device=0):
    """Time the exact-SRE sweep of an n-qubit state for several batch sizes and keep the
    fastest for later calls of that size and precision (12 <= n <= 21).  Returns
    (batch size, microseconds per X-string).  No reference counterpart."""
    return default_context(device).autotune(n, _precision(precision))


def generate_gray_table(n, q):
    """Gray table as src/Basis.jl:252-265, computed on the device.

    q == 2: (codes uint64[2^n], flips int64[2^n - 1], 1-based).
    q > 2:  (XTAB int64[n, q^n], flips int64[q^n - 1], 1-based).
    """
    if q < 2:
        raise AssertionError("Base q must be ≥ 2")
    ctx = default_context()
    return ctx.gray_table(n) if q == 2 else ctx.gray_table_general(n, q)


def load_state(path, q=2):
    """StateVec from disk (src/State.jl:388-404): .npy (numpy), otherwise whitespace-
    separated real/imaginary pairs.  With a CUDA device the file is read by hm_load_state
    straight into page-locked host memory (the state's copies to the GPU then run at full
    link speed); without one, into an ordinary numpy array with the same contents.  .jld2
    needs h5py, which this image does not ship."""
    if not path.endswith(".jld2") and _cuda_available():
        return StateVec(_native.load_state_pinned(path, q=q), q=q, copy=False)
    if path.endswith(".npy"):
        return StateVec(np.load(path), q=q)
    if path.endswith(".jld2"):
        try:
            import h5py  # noqa: F401
        except ImportError:
            raise ArgumentError(".jld2 states need h5py, which is not installed") from None
        with h5py.File(path, "r") as f:
            d = f["state"][()]
        if d.dtype.names:
            d = d[d.dtype.names[0]] + 1j * d[d.dtype.names[1]]
        return StateVec(d, q=q)
    with open(path) as f:
        vals = [float(t) for t in f.read().split()]
    if len(vals) % 2 != 0:
        raise ArgumentError("File does not contain real/imaginary pairs")
    v = np.array(vals[0::2]) + 1j * np.array(vals[1::2])
    return StateVec(v, q=q)


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def reduced_density_matrix(psi, NA, side="right", q=None, device=0):
    """rho_A = Tr_B |psi><psi| for a contiguous bipartition (src/DensityMatrix.jl:94-123),
    computed on the GPU (hm_reduced_density_matrix).

    side="right" keeps the NA most significant sites, side="left" the NA least
    significant.
    """
    s = psi if isinstance(psi, StateVec) else StateVec(psi, q=q or 2)
    if s.q not in (2, 3):
        raise ArgumentError("only q=2 and q=3 are implemented")
    if not (0 <= NA <= s.n):
        raise ArgumentError(f"need 0 ≤ NA ≤ N (got NA={NA}, N={s.n})")
    if side not in ("left", "right"):
        raise ArgumentError(f"side must be :left or :right (got {side})")
    rho = default_context(device).reduced_density_matrix(s.data, s.q, NA, side)
    return DensityMatrix(rho, q=s.q)


# ----------------------------------------------------------------------------------
# state preparation on the GPU (src/State.jl:111-374, src/Helpers.jl:102-132)

def haar_random_unitary(q, n_qudits, rng=None):
    """Haar-random unitary of size q^n x q^n (src/Helpers.jl:102-132): a complex Gaussian
    matrix, its QR factorisation, and Q with its columns rephased so that diag(R) > 0.
    Drawn with numpy's Generator; the reference draws from Julia's RNG, so the two
    streams differ."""
    if q not in (2, 3):
        raise ArgumentError("haar_random_unitary: only q=2 and q=3 are implemented")
    rng = np.random.default_rng() if rng is None else rng
    N = q ** n_qudits
    X = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    Q, R = np.linalg.qr(X)
    d = np.diag(R)
    ph = np.where(d == 0, 1.0, d / np.where(d == 0, 1.0, np.abs(d)))
    return Q * ph[None, :]


def brick_wall_pairs(n, depth):
    """Site pairs of a brick-wall circuit in layer order: odd layers (1,2),(3,4),...,
    even layers (2,3),(4,5),... (src/State.jl:172-178, 212-218)."""
    return [(s, s + 1) for layer in range(1, depth + 1) for s in range(1 if layer % 2 else 2, n, 2)]


def apply_2gate_inplace(sv, gate, s1, s2, device=0):
    """apply_2gate! (src/State.jl:254-345, 356-364): two-site gate on sites s1, s2
    (1-based, site 1 least significant), in place, on the GPU."""
    sv.data[:] = default_context(device).apply_2gate(sv.data, sv.q, gate, s1, s2)
    return sv


def apply_2gate(sv, gate, s1, s2, device=0):
    """apply_2gate (src/State.jl:366-374): as apply_2gate_inplace on a copy."""
    return apply_2gate_inplace(StateVec(sv.data.copy(), q=sv.q), gate, s1, s2, device)


def apply_brick_wall(sv, depth, gates, device=0):
    """Brick-wall circuit with the given gates (one per pair of brick_wall_pairs), in
    place, on the GPU (hm_brick_wall)."""
    sv.data[:] = default_context(device).brick_wall(sv.data, sv.q, depth, list(gates))
    return sv


def apply_brick_wall_haar(sv, depth, rng=None, device=0):
    """apply_brick_wall_haar! (src/State.jl:200-236): Haar-random two-site gates in a
    brick wall, in place."""
    gates = [haar_random_unitary(sv.q, 2, rng) for _ in brick_wall_pairs(sv.n, depth)]
    return apply_brick_wall(sv, depth, gates, device)


def rand_haar(n, depth, q=2, rng=None, device=0):
    """rand_haar (src/State.jl:111-124): |0...0> after a depth-`depth` brick wall of
    Haar-random two-site gates."""
    if q not in (2, 3):
        raise ArgumentError("rand_haar: only q=2 (qubits) and q=3 (qutrits) are implemented")
    v = np.zeros(q ** n, dtype=np.complex128)
    v[0] = 1.0
    return apply_brick_wall_haar(StateVec(v, q=q), depth, rng, device)


# one-qubit gates (each applied as kron(g, I) on the pair) and CNOT of
# apply_brick_wall_cliff! (src/State.jl:146-183), as listed there: its "H" entry is the
# identity matrix and is kept that way
_CLIFF_ONE = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0]),
              np.eye(2), np.diag([1.0, 1j])]
_CLIFF_CNOT = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=np.complex128)


def rand_cliff(n, depth=1, rng=None, device=0):
    """rand_cliff (src/State.jl:126-183): |0...0> after a brick wall whose gates are drawn
    uniformly from the six one-qubit gates (as kron(g, I)) and CNOT."""
    rng = np.random.default_rng() if rng is None else rng
    gates = []
    for _ in brick_wall_pairs(n, depth):
        k = int(rng.integers(0, len(_CLIFF_ONE) + 1))
        gates.append(np.kron(_CLIFF_ONE[k], np.eye(2)) if k < len(_CLIFF_ONE) else _CLIFF_CNOT)
    v = np.zeros(1 << n, dtype=np.complex128)
    v[0] = 1.0
    return apply_brick_wall(StateVec(v, q=2), depth, gates, device)
