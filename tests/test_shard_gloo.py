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
