"""CPU check of the ordering argument the GPU deblocker rests on.

The reference filters edge segments sequentially in CU decode order
(src/deblock.rs:687-705).  The GPU groups the segments of one pass and plane
into components -- segments on the same band whose footprints
[pos - R(mflP), pos + R(mflQ)), R(m) = 4 for m <= 3 else m + 1, overlap --
keeps reference order inside a component and runs components in any order.
Here the oracle's own segment list is replayed component by component in a
shuffled order and must reproduce the reference output bit for bit."""
import numpy as np
import pytest

import oracle
from oxideav_h266_b200 import workloads as W


def reach(m):
    return 4 if m <= 3 else m + 1


def components(log):
    keep = [i for i, r in enumerate(log) if r[8] != 0 and not (r[0] != 0 and r[5] == 1 and r[6] == 1 and r[4] != 2)]
    passes = {0: [], 1: []}
    groups = {}
    for i in keep:
        r = log[i]
        groups.setdefault((int(r[1]), int(r[0])), []).append(i)
    for (vert, plane), idxs in groups.items():
        keys = []
        for i in idxs:
            r = log[i]
            pos, band = (r[2], r[3]) if vert else (r[3], r[2])
            keys.append((band, pos - reach(r[5]), pos + reach(r[6]), i))
        keys.sort()
        j = 0
        while j < len(keys):
            k = j + 1
            end = keys[j][2]
            while k < len(keys) and keys[k][0] == keys[j][0] and keys[k][1] < end:
                end = max(end, keys[k][2])
                k += 1
            passes[0 if vert else 1].append(sorted(t[3] for t in keys[j:k]))  # emission index = reference order
            j = k
    return passes


CASES = [(s, dict(dual_tree=s % 3 == 1, tiles=s % 3 == 2, bit_depth=8 + 2 * (s % 2))) for s in range(12)]


@pytest.mark.parametrize("seed,kw", CASES)
def test_component_replay_matches_reference(seed, kw):
    pic, fa = W.stress_workload(seed, 192, 128, **kw)
    want = pic.copy()
    oracle.apply_deblocking_clipped(want, fa)
    log = oracle.deblock_edge_log(pic, fa)
    comps = components(log)
    rng = np.random.default_rng(seed)
    order = []
    for p in (0, 1):
        cs = comps[p]
        for ci in rng.permutation(len(cs)):
            order += cs[ci]
    got = pic.copy()
    oracle.deblock_replay(got, log, np.array(order, dtype=np.uint64))
    assert got.equal(want)
    assert max(len(c) for c in comps[0] + comps[1]) >= 2  # stress content forms multi-segment components
