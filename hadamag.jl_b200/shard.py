"""Multi-GPU exact SRE: one process per GPU, the Gray-code range split across ranks.

The reference splits the X-string range over MPI ranks and then over the GPUs of a
rank (ext/HadaMAGMPICUDAExt.jl:30-106) with HadaMAG.partition_counts
(src/Helpers.jl:18-23) and sums the two scalars with MPI.Allreduce.  Here every rank
computes double-double partial sums over its contiguous slice of Gray indices with the
C ABI, and the ranks exchange those partials with one all_gather (NCCL on GPUs, gloo on
CPU); every rank folds them in rank order, so all ranks get the same bits.

The sweep itself needs no other exchange: the state is replicated (2^n complex, at most
32 MiB for n <= 21) and each X-string is independent.
"""
import numpy as np


def partition_counts(n_items, parts):
    """Counts and 0-based displacements of src/Helpers.jl:18-23: the first (n mod P)
    parts get one item more."""
    base, rem = divmod(int(n_items), int(parts))
    counts = [base + 1 if i < rem else base for i in range(parts)]
    displs = [0] * parts
    for i in range(1, parts):
        displs[i] = displs[i - 1] + counts[i - 1]
    return counts, displs


def gray_slice(n, rank, world):
    """[k_begin, k_end) of Gray indices owned by `rank` of `world` for an n-qubit state."""
    counts, displs = partition_counts(1 << n, world)
    return displs[rank], displs[rank] + counts[rank]


def two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def dd_add(x, y):
    """(hi, lo) + (hi, lo) in double-double (Knuth TwoSum on the high parts)."""
    s, e = two_sum(x[0], y[0])
    lo = x[1] + y[1] + e
    hi = s + lo
    return hi, lo - (hi - s)


def dd_fold(parts):
    """Fold a sequence of (hi, lo) pairs in the given order."""
    acc = (0.0, 0.0)
    for p in parts:
        acc = dd_add(acc, (float(p[0]), float(p[1])))
    return acc


def combine_partials(gathered, n, nq):
    """gathered: array (world, 2 + 2 nq) of [p2_hi, p2_lo, m_hi, m_lo, ...] per rank.

    Returns (sre[nq], lost_norm) as src/Backends/Threads.jl:158.
    """
    g = np.asarray(gathered, dtype=np.float64).reshape(-1, 2 + 2 * nq)
    dim = float(1 << n)
    p2 = dd_fold(g[:, 0:2])
    sre = []
    for i in range(nq):
        m = dd_fold(g[:, 2 + 2 * i: 4 + 2 * i])
        sre.append(-np.log2((m[0] + m[1]) / dim))
    return np.array(sre), abs(1.0 - (p2[0] + p2[1]) / dim)


def allgather_partials(local, group=None, device=None):
    """all_gather of one rank's partial vector through torch.distributed; returns a
    (world, len) float64 numpy array in rank order."""
    import torch
    import torch.distributed as dist

    t = torch.as_tensor(np.asarray(local, dtype=np.float64), device=device)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return torch.stack(out).cpu().numpy()


def sre_sharded(compute_range, n, qs, rank, world, group=None, device=None):
    """Exact SRE over all ranks.

    compute_range(k_begin, k_end) -> (p2_dd[2], m_dd[nq, 2]) runs this rank's slice
    (the C ABI's hm_sre_range or hm_sre_range_dev).
    """
    kb, ke = gray_slice(n, rank, world)
    p2, m = compute_range(kb, ke)
    local = np.concatenate([np.asarray(p2, dtype=np.float64).reshape(2), np.asarray(m, dtype=np.float64).reshape(-1)])
    gathered = allgather_partials(local, group=group, device=device) if world > 1 else local[None, :]
    return combine_partials(gathered, n, len(qs))
