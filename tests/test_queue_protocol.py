"""A CPU model of the persistent queue sweep's protocol (csrc/sweep_queue.cuh and the
layout of csrc/queue_host.cu), run under random schedules of a handful of warps.

The model restates, in Python:
- the host layout: cost order, ring slot size, per-state X (a power of two), batches,
  global batch numbers, unit ranges, and the per-batch unit counts;
- the kernel's unit decode with a lead of L batches between a batch's pass 1 and pass 2;
- each warp's behaviour: a pipelined claim (the next unit is claimed before the current one
  runs), pass-1 units that wait for done2[q - K] before storing into slot q mod K, pass-2
  units that wait for done1[q], and the lazy announce of a finished pass-1 unit (before the
  warp's next store, before any wait, at exit).

Checked under many random interleavings: the sweep always finishes (no schedule blocks
every warp), every unit runs once, a pass-1 unit stores into a slot only after every
pass-2 unit of the slot's previous batch has read it, and a pass-2 unit reads only after
every pass-1 unit of its batch has announced.  The same model with the earlier wait target
(the current state's unit count instead of the slot's previous batch's) violates the slot
rule on batches of different sizes, which is the failure this rule fixes."""
import random

import pytest


def layout(items, x_slot):
    """items: (n, kb, ke).  x_slot: X-strings per ring slot of the largest two-pass state
    (the host's tuned or slot-size rule).  Returns (states, total units, bunits)."""
    order = sorted(range(len(items)), key=lambda i: (items[i][0] < 12, -((items[i][2] - items[i][1]) * 2.0 ** items[i][0])))
    nmax = max([n for n, kb, ke in items if n >= 12 and ke > kb] or [0])
    slot_elems = 0
    if nmax:
        X = x_slot
        while X & (X - 1):
            X &= X - 1
        slot_elems = X << (nmax - 1)
    states, total, qnext, bunits = [], 0, 0, []
    for oi in order:
        n, kb, ke = items[oi]
        s = dict(n=n, kb=kb, ke=ke, u0=total, X=0, lgX=0, nbatch=0, q0=0)
        length = ke - kb
        if length > 0:
            if n <= 11:
                s["X"] = 1 << (11 - n)
                total += (length + s["X"] - 1) // s["X"]
            else:
                xcap = slot_elems >> (n - 1)
                x = 1
                while x < length and x < xcap:
                    x <<= 1
                s["X"], s["lgX"] = x, x.bit_length() - 1
                s["nbatch"] = (length + x - 1) // x
                s["q0"] = qnext
                qnext += s["nbatch"]
                U = x << (n - 11)
                bunits += [U] * s["nbatch"]
                total += 2 * s["nbatch"] * U
        s["u1"] = total
        states.append(s)
    return states, total, bunits


def decode(s, p, lead):
    """(batch, pass, unit within the batch) of unit p of a two-pass state, as the kernel."""
    hi = s["n"] - 11
    lgU = s["lgX"] + hi
    U = 1 << lgU
    L, nb = lead, s["nbatch"]
    za = min(L, nb)
    A = za << lgU
    B = max(nb - L, 0) << (lgU + 1)
    if p < A:
        return p >> lgU, 1, p & (U - 1)
    if p < A + B:
        p2 = p - A
        sg = L + (p2 >> (lgU + 1))
        w = p2 & (2 * U - 1)
        return (sg if w < U else sg - L), (1 if w < U else 2), w & (U - 1)
    p3 = p - A - B
    sg = max(L, nb) + (p3 >> lgU)
    return sg - L, 2, p3 & (U - 1)


class Violation(Exception):
    pass


def simulate(items, K, lead, nwarps, x_slot, seed, target="batch"):
    """One random schedule.  target: "batch" (the kernel's rule: batch q - K's own unit
    count) or "current" (the earlier rule: the current state's count)."""
    states, total, bunits = layout(items, x_slot)
    rng = random.Random(seed)
    nq = len(bunits)
    done1, done2, reads = [0] * nq, [0] * nq, [0] * nq
    owner = [None] * K
    ran = [0] * total
    nxt = [0]

    def claim():
        c = nxt[0]
        nxt[0] += 1
        return c

    def warp():
        pending = [None]

        def announce():
            if pending[0] is not None:
                done1[pending[0]] += 1
                pending[0] = None

        c = claim()
        while True:
            u = c
            if u >= total:
                break
            c = claim()  # the next claim is in flight while this unit runs
            yield ("step",)
            s = next(st for st in states if st["u0"] <= u < st["u1"])
            ran[u] += 1
            if s["n"] <= 11:
                continue
            b, ps, r = decode(s, u - s["u0"], lead)
            q = s["q0"] + b
            U = s["X"] << (s["n"] - 11)
            xs = r & (s["X"] - 1)
            active = s["kb"] + b * s["X"] + xs < s["ke"]
            if ps == 1:
                if q >= K:
                    announce()
                    need = bunits[q - K] if target == "batch" else U
                    yield ("wait", lambda q=q, need=need: done2[q - K] >= need)
                    if reads[q - K] != bunits[q - K]:
                        raise Violation(f"batch {q} stores into slot {q % K} while batch {q - K} "
                                        f"has {reads[q - K]} of {bunits[q - K]} reads done")
                owner[q % K] = q
                yield ("step",)
                if active:
                    announce()
                    pending[0] = q  # announced once its stores have completed
                else:
                    announce()
                    done1[q] += 1
            else:
                announce()
                yield ("wait", lambda q=q, U=U: done1[q] >= U)
                if owner[q % K] != q:
                    raise Violation(f"batch {q} reads slot {q % K} holding batch {owner[q % K]}")
                reads[q] += 1
                yield ("step",)
                done2[q] += 1
        announce()

    gens = [warp() for _ in range(nwarps)]
    cur = [next(g, None) for g in gens]
    while any(a is not None for a in cur):
        runnable = [i for i, a in enumerate(cur) if a is not None and (a[0] == "step" or a[1]())]
        if not runnable:
            raise Violation("every unfinished warp waits: deadlock")
        i = rng.choice(runnable)
        cur[i] = next(gens[i], None)
    assert ran == [1] * total, "every unit runs exactly once"
    assert all(done1[q] == bunits[q] and done2[q] == bunits[q] for q in range(nq))
    return total


CASES = [
    # (items, K, lead, x_slot): mixed sizes in one queue
    ([(14, 0, 1), (13, 0, 1), (12, 0, 1), (12, 0, 1), (12, 0, 1)], 2, 1, 1),  # FP32 x = 0 batches
    ([(13, 0, 40), (12, 0, 24), (9, 0, 512), (12, 5, 9)], 3, 2, 4),
    ([(14, 0, 17), (13, 0, 33), (12, 0, 70)], 4, 2, 2),
    ([(12, 0, 64)], 2, 1, 8),
    ([(13, 3, 50), (13, 0, 2), (12, 0, 3), (8, 0, 256)], 3, 1, 4),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_queue_protocol_random_schedules(case):
    items, K, lead, x_slot = CASES[case]
    for seed in range(60):
        for nwarps in (2, 5, 9):
            simulate(items, K, lead, nwarps, x_slot, 1000 * case + 17 * seed + nwarps)


def test_lead_decode_covers_every_unit_once():
    for lead in range(1, 6):
        for nb in range(1, 9):
            for lgx in range(0, 3):
                s = dict(n=12, lgX=lgx, nbatch=nb)
                U = (1 << lgx) << 1
                got = [decode(s, p, lead) for p in range(2 * nb * U)]
                assert sorted(got) == sorted((b, ps, r) for b in range(nb) for ps in (1, 2) for r in range(U))
                pos = {g: i for i, g in enumerate(got)}
                for b in range(nb):
                    assert pos[(b, 2, 0)] > pos[(b, 1, U - 1)]  # a batch's pass 2 after all of its pass 1


def test_current_state_target_breaks_slot_reuse():
    """With the earlier wait target, batches of different sizes (the FP32 x = 0 batches of
    2^(n - 11) units) let a slot be rewritten before its previous batch was read."""
    items, K, lead, x_slot = CASES[0]
    hit = 0
    for seed in range(400):
        try:
            simulate(items, K, lead, 4, x_slot, seed, target="current")
        except Violation as e:
            assert "stores into slot" in str(e)
            hit += 1
    assert hit > 0
