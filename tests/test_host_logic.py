"""Host-side logic that needs no GPU: the autotuner's search and the serving
stream generator."""
import numpy as np

from indexingpu_b200 import autotune
from indexingpu_b200 import workload as wl


def test_autotune_coordinate_descent_picks_the_best():
    # A made-up cost surface: best at find tile 8, write tile 32, bucketing
    # on, 6 blocks per SM.
    def score(c):
        s = 100.0 - abs(c["find_tile"] - 8) - (0 if c["write_tile"] == 32 else 7) + (3 if c["bucketing"] else 0)
        s -= 0 if c["form"] == "forked" else 5
        b = c["blocks_per_sm"] or 8
        return s - abs(b - 6)

    cases = []

    def make_case(i):
        cases.append(i)
        return {"i": i}

    seen = []

    def trial(tree, case, config, stream):
        seen.append((case["i"], dict(config)))
        return score(config)

    best, trials = autotune.tune(None, make_case, trial=trial)
    assert (best["find_tile"], best["write_tile"], best["bucketing"], best["blocks_per_sm"]) == (8, 32, True, 6)
    assert best["form"] == "forked"
    # forked and persistent x 4 find tiles x 2 write tiles x bucketing, grouped
    # (no buckets) x 4 x 2, then blocks per SM x 8.
    assert len(trials) == 2 * 4 * 2 * 2 + 4 * 2 + 8
    assert not any(t["form"] == "grouped" and t["bucketing"] for t in trials)
    # One warm-up case for all 24 kernel flavours, then a fresh case per trial.
    assert cases == list(range(len(trials) + 1))
    assert sum(1 for i, _ in seen if i == 0) == 24
    assert best["mops"] == max(t["mops"] for t in trials)


def test_serve_stream_shapes_and_disjoint_keys():
    c2 = wl.C2(n_preload=20000, n_prefixes=32)
    st = wl.serve_stream(c2, 300, rate_per_s=1e5, min_ops=1, max_ops=64, disjoint=True, seed=7)
    n_ops = int(st["nops"].sum())
    assert len(st["types"]) == n_ops == len(st["keys"])
    assert st["nops"].min() >= 1 and st["nops"].max() <= 64
    assert np.array_equal(st["first"], np.concatenate([[0], np.cumsum(st["nops"][:-1])]))
    assert np.all(np.diff(st["arrival_ns"].astype(np.int64)) >= 0)
    # Every op touches its own key.
    assert len(np.unique(st["ids"])) == n_ops
    assert len(np.unique(st["keys"][:, :], axis=0)) == n_ops
    # Finds carry no value; inserts use fresh ids.
    f = st["types"] == wl.REQ_FIND
    assert (st["vlens"][f] == 0).all()
    assert (st["ids"][st["types"] == wl.REQ_INSERT] >= c2.n_preload).all()


def test_serve_stream_op_seed_keeps_sizes():
    c2 = wl.C2(n_preload=20000, n_prefixes=32)
    a = wl.serve_stream(c2, 50, min_ops=8, max_ops=512, seed=0xC4, op_seed=1, first_fresh=30000)
    b = wl.serve_stream(c2, 50, min_ops=8, max_ops=512, seed=0xC4, op_seed=2, first_fresh=30000)
    assert np.array_equal(a["nops"], b["nops"])
    assert not np.array_equal(a["types"], b["types"])
    # Burst arrivals.
    assert (a["arrival_ns"] == 0).all()
