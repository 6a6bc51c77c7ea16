"""Host check of the group sum inside a warp that the streaming deposit on the Fourier y grid uses
(gem-pic-3d_b200/csrc/k_plasma.cu, sdeposit_warp): lanes with equal keys form a group; every round each lane of
even rank in its group adds the value of the next remaining member above it (a shuffle from that lane) and the
lanes of odd rank leave, until no lane has a member above it. The steps are restated here lane by lane with the
device function's 32-bit masks, and the lowest lane of every group must end with the exact sum of its group (integer
values), for groupings from all-distinct to one group of 32, contiguous and interleaved."""
import math
import random

import pytest

FULL = 0xFFFFFFFF


def warp_group_sum(keys, vals):
    lanes = range(32)
    peers = [sum(1 << j for j in lanes if keys[j] == keys[i]) for i in lanes]
    rank0 = [bin(peers[i] & ((1 << i) - 1)).count("1") for i in lanes]
    above = [peers[i] & ~(((2 << i) - 1) & FULL) & FULL for i in lanes]     # (2u << 31) - 1u wraps to all ones
    rank, a, rounds = rank0[:], list(vals), 0
    while any(above):                                                      # __any_sync(above != 0)
        nxt = [(above[i] & -above[i]).bit_length() - 1 if above[i] else i for i in lanes]   # __ffs - 1
        take = [above[i] != 0 and not (rank[i] & 1) for i in lanes]
        t = [a[nxt[i]] for i in lanes]                                     # __shfl_sync reads before any add
        a = [a[i] + t[i] if take[i] else a[i] for i in lanes]
        gone = sum(1 << i for i in lanes if rank[i] & 1)                   # __ballot_sync(rank & 1)
        above = [0 if rank[i] & 1 else above[i] & ~gone & FULL for i in lanes]
        rank = [r >> 1 for r in rank]
        rounds += 1
    return a, rank0, rounds


def groupings():
    rng = random.Random(7)
    yield list(range(32))                                   # no sharing
    yield [0] * 32                                          # one group
    yield [i // 4 for i in range(32)]                       # contiguous groups of four (lattice order)
    yield [i % 3 for i in range(32)]                        # interleaved
    yield [i // 2 if i < 16 else 100 + i for i in range(32)]
    for alphabet in (2, 3, 5, 8, 12, 20):
        for _ in range(40):
            yield [rng.randrange(alphabet) for _ in range(32)]
    for _ in range(40):                                     # inactive lanes: keys unique to each
        yield [rng.randrange(4) if rng.random() < 0.6 else -1 - i for i in range(32)]


@pytest.mark.parametrize("case", list(range(5)) + [None])
def test_lowest_lane_of_every_group_holds_its_sum(case):
    rng = random.Random(11)
    cases = list(groupings())
    for keys in (cases if case is None else [cases[case]]):
        vals = [rng.randrange(1, 1 << 20) for _ in range(32)]
        a, rank0, rounds = warp_group_sum(keys, vals)
        sizes = {}
        for k in keys:
            sizes[k] = sizes.get(k, 0) + 1
        for i in range(32):
            if rank0[i] == 0:
                assert a[i] == sum(v for k, v in zip(keys, vals) if k == keys[i]), (keys, i)
        assert rounds <= math.ceil(math.log2(max(sizes.values()))), (keys, rounds)
