"""Exact FP32 path at the largest configured sizes, against the oracle
restatement of utils.h:80-158 (itself pinned to the compiled reference by
test_oracle.py): ids and distances bit for bit.

The screen keeps a row only if its FP32 screening distance, widened by the
rigorous error margin of screen_eps, can still reach the running k-th bound;
these tests check that argument where it is hardest -- N = 1e7 rows, slabs
up to the whole base, and queries with fewer than 100 passing rows -- and
the plain configuration whole (every one of its 1e4 queries).
"""
import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu
UMAX = 0xFFFFFFFF


def test_config1_whole():
    """N = 1e5, all Q = 1e4 queries of the plain configuration, one batch."""
    vecs, labels, ts, q, metas = datagen.make_workload(1)
    assert q.shape[0] == 10_000
    with fknn.Index(vecs, labels, ts) as idx:
        ids, dists, st = idx.search(q, metas, return_stats=True)
    oids, odists = oracle.exact_knn(vecs, labels, ts, q, metas)
    bad = np.nonzero(np.any(ids != oids, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of 10000 queries differ, first {bad[:5]}"
    np.testing.assert_array_equal(dists.view(np.uint32), odists.view(np.uint32))
    # the configuration has queries with fewer than 100 passing rows: padded
    assert (ids == UMAX).any()


def pick_queries(counts, types, rng, n_random=256):
    """Indices of a checked sample: the 32 largest slabs, up to 32 queries
    with fewer than 100 passing rows (or the smallest slabs), and a random
    draw of n_random stratified by query type."""
    order = np.argsort(counts, kind="stable")
    largest = order[-32:]
    short = np.nonzero(counts < 100)[0]
    short = short[:32] if len(short) else order[:32]
    rest = []
    for t in range(4):
        pool = np.nonzero(types == t)[0]
        rest.append(rng.choice(pool, size=min(len(pool), n_random // 4), replace=False))
    return np.unique(np.concatenate([largest, short] + rest))


@pytest.mark.parametrize("cfg", [3, 4])
def test_n1e7_sampled_bitexact(cfg):
    """N = 1e7 (configurations 3 and 4): a batch of 20,000 of the
    configuration's queries is searched together, and >= 256 of them --
    every query type, the largest slabs (the whole base for type 0; the
    38 % category under Zipf 1.5) and queries with fewer than 100 passing
    rows -- are compared with the oracle bit for bit."""
    vecs, labels, ts, q, metas = datagen.make_workload(cfg, nq=20_000)
    counts = oracle.count_matches_sorted(labels, ts, metas)
    sel = pick_queries(counts, metas[:, 0].astype(np.int64), np.random.default_rng(100 + cfg))
    assert len(sel) >= 256
    with fknn.Index(vecs, labels, ts) as idx:
        ids, dists, st = idx.search(q, metas, return_stats=True)
    # every result sorted ascending with +inf padding last, padding iff short
    valid = ids != UMAX
    assert np.all(dists[:, 1:] >= dists[:, :-1])
    np.testing.assert_array_equal(valid.sum(axis=1), np.minimum(counts, 100))
    oids, odists = oracle.exact_knn(vecs, labels, ts, q[sel], metas[sel])
    bad = np.nonzero(np.any(ids[sel] != oids, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of {len(sel)} sampled queries differ, first {sel[bad[:5]]}"
    np.testing.assert_array_equal(dists[sel].view(np.uint32), odists.view(np.uint32))
    # the checked sample reaches both ends of the selectivity range
    assert counts[sel].max() >= 0.3 * vecs.shape[0]
    assert counts[sel].min() < 100 or cfg == 3
