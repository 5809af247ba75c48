"""Host model of the chunk-major near-field walk (k_leaf_units_flat in
jaccpot_b200/csrc/fmm_kernels.cuh): the invariants the kernel relies on, for
every leaf occupancy it takes (17..32 targets) and source-chunk counts
1..64.

  * lane l of step s holds item f = 32 s + l = c * nt + t; the kernel's
    incremental update (t += 32 - nt, c += 1, one wrap) equals divmod;
  * a step spans at most three consecutive chunks, so a ring of four chunk
    slots, refilled before the step's compute, never overwrites a chunk the
    step reads;
  * within a step a target appears at most twice, at lanes l < nt and l + nt
    (the partner holding the next chunk), so lanes < nt own distinct targets;
  * applying, per step, lane l's partial and then its partner's gives every
    target each of its chunks exactly once, in chunk order -- the order of
    the lane-per-target form, hence the same compensated sums."""

from __future__ import annotations

import pytest


def walk(nt: int, C: int):
    total = nt * C
    c = [1 if lane >= nt else 0 for lane in range(32)]
    t = [lane - c[lane] * nt for lane in range(32)]
    staged = 0
    ring = {}
    adds = {k: [] for k in range(nt)}
    for base in range(0, total, 32):
        chi = min(c[31], C - 1)
        while staged <= chi:  # stage chunk `staged` into slot staged % 4
            ring[staged % 4] = staged
            staged += 1
        items = {}
        for lane in range(32):
            f = base + lane
            assert (c[lane], t[lane]) == divmod(f, nt)
            if f < total:
                assert ring[c[lane] % 4] == c[lane], "a chunk the step reads was overwritten"
                items[lane] = (t[lane], c[lane])
        span = {cc for _, cc in items.values()}
        assert max(span) - min(span) <= 2
        owners = [items[l][0] for l in range(nt) if l in items]
        assert len(owners) == len(set(owners))
        for lane in range(nt):
            if lane not in items:
                continue
            tt, cc = items[lane]
            adds[tt].append(cc)
            if lane + nt < 32 and (lane + nt) in items:
                assert items[lane + nt] == (tt, cc + 1)
                adds[tt].append(cc + 1)
        for lane in range(nt, 32):  # every item at lanes >= nt is some lane < nt's partner
            if lane in items:
                assert items[lane - nt][0] == items[lane][0]
        for lane in range(32):
            t[lane] += 32 - nt
            c[lane] += 1
            if t[lane] >= nt:
                t[lane] -= nt
                c[lane] += 1
    return adds


@pytest.mark.parametrize("nt", range(17, 33))
def test_chunk_major_walk_invariants(nt):
    for C in range(1, 65):
        adds = walk(nt, C)
        for tt in range(nt):
            assert adds[tt] == list(range(C)), (nt, C, tt)
