"""Multi-rank exact SRE on CPU: two gloo ranks split the Gray range exactly as the
GPU ranks do (hadamag_b200.shard) and exchange double-double partials with
all_gather; each rank's slice is evaluated by the oracle, the combined result must
equal the single-process value."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, rand_state


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, q, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import hadamag_b200 as hm
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    psi = rand_state(1 << n, 31)

    def compute_range(kb, ke):
        p2, m = O.sre_sums(psi, q, kb + 1, ke, nthreads=2)  # oracle uses 1-based inclusive ranges
        return np.array([p2, 0.0]), np.array([[m, 0.0]])

    sre, lost = hm.shard.sre_sharded(compute_range, n, (q,), rank, world)
    out[rank] = (float(sre[0]), float(lost))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_sre_matches_single(world, oracle):
    n, q = 9, 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, n, q, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    ref, ref_lost = oracle.sre(rand_state(1 << n, 31), q)
    for r in range(world):
        assert res[r][0] == pytest.approx(ref, rel=1e-13)
        assert res[r][0] == res[0][0]  # every rank folds the partials in the same order


def test_gray_slices_cover_range(hm):
    for n in range(0, 12):
        for world in range(1, 9):
            sl = [hm.shard.gray_slice(n, r, world) for r in range(world)]
            assert sl[0][0] == 0 and sl[-1][1] == 1 << n
            assert all(sl[i][1] == sl[i + 1][0] for i in range(world - 1))


def test_dd_fold_order_stable(hm):
    rng = np.random.default_rng(0)
    parts = [(float(v), 0.0) for v in rng.normal(size=1000) * 10.0 ** rng.integers(-8, 8, size=1000)]
    a = hm.shard.dd_fold(parts)
    b = hm.shard.dd_fold(parts[::-1])
    assert a[0] + a[1] == b[0] + b[1]


# ----------------------------------------------------------------------------------
# MC chains, Mana X-string ranges and batched state lists across gloo ranks

def _mc_stream(n, nbeta, nsamples):
    rng = np.random.default_rng(7)
    pd = rng.integers(1, 1 << n, size=(nbeta, nsamples), dtype=np.uint64)
    rs = rng.random((nbeta, nsamples))
    return pd, rs


def _batched_states():
    ns = [3, 7, 5, 8, 4, 6, 2]
    return ns, [rand_state(1 << n, 60 + i) for i, n in enumerate(ns)]


def _kind_worker(kind, rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import hadamag_b200 as hm
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    if kind == "mc":
        n, q, nbeta, nsamples = 6, 2, 5, 40
        psi = rand_state(1 << n, 41)
        pd, rs = _mc_stream(n, nbeta, nsamples)

        def compute_chains(cb, ce):
            o = [O.mc_sre_beta(psi, q, i / (nbeta - 1), pd[i], rs[i])[0] for i in range(cb, ce)]
            return np.array([x[0] for x in o]), np.array([x[2] for x in o]), np.array([x[3] for x in o])

        m2, M2, M2ADD, P2 = hm.shard.mc_sharded(compute_chains, nbeta, rank, world)
        out[rank] = (float(m2), [float(v) for v in M2])
    elif kind == "mana":
        L = 5
        psi = rand_state(3 ** L, 51)

        def compute_range(xb, xe):
            return (O.mana_sum(psi, xb + 1, xe, nthreads=1), 0.0)

        out[rank] = float(hm.shard.mana_sharded(compute_range, L, rank, world))
    else:
        ns, states = _batched_states()

        def compute(idx):
            vals = np.array([[O.sre(states[i], 2)[0], O.sre(states[i], 3)[0]] for i in idx])
            return vals, np.array([O.sre(states[i], 2)[1] for i in idx])

        vals, lost = hm.shard.batched_sharded(compute, ns, 2, rank, world)
        out[rank] = [list(map(float, r)) for r in vals]
    dist.destroy_process_group()


def _run_kind(kind, world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_kind_worker, args=(kind, r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        return dict(out)


@pytest.mark.parametrize("world", [2, 3])
def test_mc_chains_sharded_match_single(world, oracle):
    n, q, nbeta, nsamples = 6, 2, 5, 40
    pd, rs = _mc_stream(n, nbeta, nsamples)
    m2, M2, _, _ = oracle.mc_sre(rand_state(1 << n, 41), q, nbeta, nsamples, pd.reshape(-1), rs.reshape(-1))
    res = _run_kind("mc", world)
    for r in range(world):
        assert res[r][1] == pytest.approx(list(M2), rel=1e-14)
        assert res[r][0] == pytest.approx(m2, rel=1e-13)
        assert res[r][0] == res[0][0]


@pytest.mark.parametrize("world", [2, 4])
def test_mana_sharded_matches_single(world, oracle):
    ref = oracle.mana_pure(rand_state(3 ** 5, 51))
    res = _run_kind("mana", world)
    for r in range(world):
        assert res[r] == pytest.approx(ref, rel=1e-12)
        assert res[r] == res[0]


@pytest.mark.parametrize("world", [2, 4])
def test_batched_sharded_matches_single(world, oracle):
    ns, states = _batched_states()
    res = _run_kind("batched", world)
    for r in range(world):
        for i, s in enumerate(states):
            assert res[r][i][0] == pytest.approx(oracle.sre(s, 2)[0], rel=1e-13)
            assert res[r][i][1] == pytest.approx(oracle.sre(s, 3)[0], rel=1e-13)


def test_balance_states_covers_every_state(hm):
    for world in (1, 2, 3, 5):
        ns = list(np.random.default_rng(world).integers(8, 19, size=37))
        parts = hm.shard.balance_states(ns, world)
        assert sorted(i for p in parts for i in p) == list(range(len(ns)))
        loads = [sum(4.0 ** ns[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= 4.0 ** max(ns)
