"""Multi-GPU runs: one process per GPU.

Exact SRE splits the Gray-code range across ranks; MC_SRE splits its beta chains;
pure-state Mana splits its ternary X-string range; batched SRE splits its list of
states by cost.

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


def dd_fold_rows(gathered):
    """Fold the per-rank rows [p2_hi, p2_lo, m_hi, m_lo, ...] in rank order; returns one
    row of the same layout."""
    g = np.asarray(gathered, dtype=np.float64)
    g = g.reshape(-1, g.shape[-1])
    out = np.zeros(g.shape[1])
    for j in range(0, g.shape[1], 2):
        out[j:j + 2] = dd_fold(g[:, j:j + 2])
    return out


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


# ----------------------------------------------------------------------------------
# padded all_gather of per-rank tables with different row counts

def allgather_rows(rows, max_rows, group=None, device=None, world=1):
    """all_gather of a (k, w) float64 table, k <= max_rows, padded with NaN; returns the
    list of each rank's k rows in rank order (one collective of fixed size)."""
    rows = np.asarray(rows, dtype=np.float64)
    if rows.ndim == 1:
        rows = rows[:, None]
    w = rows.shape[1]
    buf = np.full((max_rows + 1, w), np.nan)
    buf[0, 0] = rows.shape[0]  # row 0 carries the count
    buf[1:1 + rows.shape[0]] = rows
    g = allgather_partials(buf.reshape(-1), group=group, device=device) if world > 1 else buf.reshape(1, -1)
    out = []
    for r in range(g.shape[0]):
        t = g[r].reshape(max_rows + 1, w)
        out.append(t[1:1 + int(t[0, 0])])
    return out


# ----------------------------------------------------------------------------------
# MC_SRE: independent beta chains (src/Backends/Threads.jl:161-221)

def chain_slice(nbeta, rank, world):
    """[chain_begin, chain_end) of the beta grid owned by `rank`."""
    counts, displs = partition_counts(nbeta, world)
    return displs[rank], displs[rank] + counts[rank]


def mc_combine(M2, M2ADD):
    """m2 = -log2(2^-I + I_add) with I, I_add the composite Simpson integrals over the
    uniform beta grid on [0, 1] (src/Helpers.jl:223-236, src/Backends/Threads.jl:207-220),
    summed in the same order as hm_mc_sre's device combination."""
    M2 = np.asarray(M2, dtype=np.float64)
    M2ADD = np.asarray(M2ADD, dtype=np.float64)
    nb = M2.size
    if nb < 3 or nb % 2 != 1:
        raise ValueError("Simpson needs an odd number of beta points >= 3")
    h = 1.0 / (nb - 1)
    odd = even = odda = evena = 0.0
    for i in range(1, nb - 1):
        if i % 2 == 1:
            odd += float(M2[i])
            odda += float(M2ADD[i])
        else:
            even += float(M2[i])
            evena += float(M2ADD[i])
    I_res = (h / 3.0) * (float(M2[0]) + float(M2[-1]) + 4.0 * odd + 2.0 * even)
    I_add = (h / 3.0) * (float(M2ADD[0]) + float(M2ADD[-1]) + 4.0 * odda + 2.0 * evena)
    return -np.log2(2.0 ** (-I_res) + I_add)


def mc_sharded(compute_chains, nbeta, rank, world, group=None, device=None):
    """MC_SRE over all ranks.  compute_chains(chain_begin, chain_end) -> (M2, M2ADD, P2)
    for this rank's chains (the C ABI's hm_mc_sre_chains).  Returns
    (m2, M2[nbeta], M2ADD[nbeta], P2[nbeta]) on every rank."""
    cb, ce = chain_slice(nbeta, rank, world)
    if ce > cb:
        M2, M2ADD, P2 = compute_chains(cb, ce)
        local = np.stack([np.asarray(M2), np.asarray(M2ADD), np.asarray(P2)], axis=1)
    else:
        local = np.zeros((0, 3))
    per_rank = allgather_rows(local, -(-nbeta // world), group=group, device=device, world=world)
    allc = np.concatenate(per_rank, axis=0)
    return mc_combine(allc[:, 0], allc[:, 1]), allc[:, 0], allc[:, 1], allc[:, 2]


# ----------------------------------------------------------------------------------
# Mana of a pure state: X-string range split (src/Backends/Threads.jl:223-271)

def mana_sharded(compute_range, L, rank, world, group=None, device=None):
    """Mana over all ranks.  compute_range(x_begin, x_end) -> (hi, lo) double-double
    sum of |W| over this rank's X-strings (the C ABI's hm_mana_pure_range)."""
    counts, displs = partition_counts(3 ** L, world)
    xb, xe = displs[rank], displs[rank] + counts[rank]
    local = np.asarray(compute_range(xb, xe) if xe > xb else (0.0, 0.0), dtype=np.float64).reshape(2)
    gathered = allgather_partials(local, group=group, device=device) if world > 1 else local[None, :]
    S = dd_fold(gathered)
    return np.log2(S[0] + S[1]) / np.log2(3.0)


# ----------------------------------------------------------------------------------
# batched SRE: the list of states split by cost

def balance_states(ns, world):
    """Deterministic split of states with qubit counts ns over `world` ranks: largest
    first (4^n work each), each to the least loaded rank (lowest rank on ties).
    Returns one sorted index list per rank."""
    order = sorted(range(len(ns)), key=lambda i: (-int(ns[i]), i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += 4.0 ** int(ns[i])
    return [sorted(p) for p in parts]


def batched_sharded(compute, ns, nq, rank, world, group=None, device=None):
    """SRE of many states over all ranks.  compute(indices) -> (vals[len, nq], lost[len])
    for this rank's states (the C ABI's hm_sre_batched).  Returns (vals[S, nq], lost[S])
    in input order on every rank."""
    parts = balance_states(ns, world)
    mine = parts[rank]
    if mine:
        vals, lost = compute(mine)
        local = np.concatenate([np.asarray(vals, dtype=np.float64).reshape(len(mine), nq),
                                np.asarray(lost, dtype=np.float64).reshape(len(mine), 1)], axis=1)
    else:
        local = np.zeros((0, nq + 1))
    per_rank = allgather_rows(local, max(len(p) for p in parts), group=group, device=device, world=world)
    vals = np.zeros((len(ns), nq))
    lost = np.zeros(len(ns))
    for r, rows in enumerate(per_rank):
        for j, i in enumerate(parts[r]):
            vals[i] = rows[j, :nq]
            lost[i] = rows[j, nq]
    return vals, lost
