"""mt_serve: the device-resident request loop.

Every op of the streams below touches its own key (workload.serve_stream with
disjoint=True), so each op's result is defined independently of how requests
interleave: the CPU oracle applied to the whole stream as one mixed batch
gives the expected result of every op.  The same stream is served (a) in the
plain form, one request alone at a time, and (b) by the device-resident loop
with many requests in flight together; both must equal the oracle op by op and
leave the same contents.
"""
import numpy as np
import pytest

from indexingpu_b200 import workload as wl
from indexes import OracleIndex

pytestmark = pytest.mark.gpu
MAXK, MAXV = 16, 8
N_PRE = 40000


def _tree(torch, c2, tile=8, write_tile=32, pool_bytes=256 << 20):
    from indexingpu_b200 import GpuMasstree
    keys, lens, vals, vlens = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c2.keys(np.arange(N_PRE)))
    t = GpuMasstree(pool_bytes=pool_bytes, tile_size=tile)
    t.set_write_tile_size(write_tile)
    t.insert(keys, MAXK, lens, vals, MAXV, vlens, N_PRE)
    t.sync()
    return t


def _expected(c2, st):
    o = OracleIndex()
    k, l, v, vl = c2.keys(np.arange(N_PRE))
    o.insert(k, l, v, vl)
    vals, vlens, res = o.mixed(st["types"], st["keys"], st["lens"], st["vals"], st["vlens"])
    return o, vals, vlens, res


def _serve(torch, tree, st, **kw):
    dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in ("types", "keys", "lens", "vals", "vlens")}
    n = len(st["types"])
    results = torch.zeros(n, dtype=torch.bool, device="cuda")
    lat, stats = tree.serve(dev["types"], dev["keys"], MAXK, dev["lens"], dev["vals"], MAXV, dev["vlens"], results,
                            st["first"], st["nops"], st["arrival_ns"], **kw)
    tree.sync()
    return lat, stats, dev["vals"].cpu().numpy(), dev["vlens"].cpu().numpy(), results.cpu().numpy()


def _check(st, got, exp):
    _, _, gv, gvl, gres = got
    _, ev, evl, eres = exp
    find = st["types"] == wl.REQ_FIND
    np.testing.assert_array_equal(gres[~find].astype(np.uint8), eres[~find])
    np.testing.assert_array_equal(gvl[find], evl[find])
    for i in np.nonzero(find & (evl > 0))[0]:
        c = min(int(evl[i]), MAXV)
        assert np.array_equal(gv[i, :c], ev[i, :c]), i


def _dump(torch, tree, n):
    lower = torch.zeros((1, MAXK), dtype=torch.uint32, device="cuda")
    lens = torch.ones(1, dtype=torch.uint32, device="cuda")
    counts = torch.zeros(1, dtype=torch.uint32, device="cuda")
    vals = torch.zeros((1, n, MAXV), dtype=torch.uint32, device="cuda")
    vlens = torch.zeros((1, n), dtype=torch.uint32, device="cuda")
    keys = torch.zeros((1, n, MAXK), dtype=torch.uint32, device="cuda")
    klens = torch.zeros((1, n), dtype=torch.uint32, device="cuda")
    tree.scan(lower, lens, MAXK, n, 1, counts=counts, values=vals, max_value_length=MAXV, value_lengths=vlens,
              out_keys=keys, out_key_lengths=klens)
    tree.sync()
    c = int(counts[0])
    return [x[0, :c].cpu().numpy() for x in (keys, klens, vals, vlens)]


@pytest.mark.parametrize("tile,write_tile,rate,chunk", [(8, 32, None, 0), (8, 16, 2e5, 8), (16, 32, 5e4, 32),
                                                        (4, 16, 2e5, 1)])
def test_served_equals_alone(tile, write_tile, rate, chunk):
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    st = wl.serve_stream(c2, 1500, rate_per_s=rate, disjoint=True, seed=0xC5 + tile + write_tile)
    exp = _expected(c2, st)
    plain_tree, served_tree = _tree(torch, c2, tile, write_tile), _tree(torch, c2, tile, write_tile)
    try:
        plain = _serve(torch, plain_tree, st, plain=True)
        served = _serve(torch, served_tree, st, chunk_ops=chunk, epoch_us=5000)
        n_ops = int(st["nops"].sum())
        for got in (plain, served):
            assert got[1]["requests_done"] == len(st["nops"])
            assert got[1]["ops_done"] == n_ops
            assert (got[0] > 0).all()
            _check(st, got, exp)
        # Identical contents after the stream, equal to the oracle's.
        n_final = N_PRE + n_ops
        a, b = _dump(torch, plain_tree, n_final), _dump(torch, served_tree, n_final)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
        ok, nkeys, report = served_tree.validate()
        assert ok, report
        assert nkeys == len(a[0]) == len(exp[0].dump(MAXK, MAXV)[0])
    finally:
        plain_tree.close()
        served_tree.close()


def test_served_admission_waits_for_memory():
    """A budget just above the tree's footprint admits few requests at a time;
    admission waits for completions and reclaimed slabs, and every request
    still completes with the oracle's results."""
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    # Mostly updates (their old chains come back at every reclaim), few inserts
    # (the tree grows by about 1.5 slabs per insert).
    st = wl.serve_stream(c2, 600, rate_per_s=None, disjoint=True, seed=0x5E, mix=(0.5, 0.1, 0.3, 0.1))
    exp = _expected(c2, st)
    tree = _tree(torch, c2, 8, 32, pool_bytes=64 << 20)
    try:
        s = tree.stats()
        total = s["total_slabs"]
        held = s["used_slabs"] + s["limbo_slabs"]
        # The admission estimate is 2 slabs per insert or update (16-slice keys,
        # 8-slice values); allow half the stream's estimate above what the
        # tree holds, so the burst at time 0 cannot be admitted at once.
        writes = int(np.isin(st["types"], [wl.REQ_INSERT, wl.REQ_UPDATE]).sum())
        budget = (held + writes) / total
        got = _serve(torch, tree, st, chunk_ops=8, epoch_us=500, memory_budget=budget)
        assert got[1]["requests_done"] == len(st["nops"])
        assert got[1]["admission_waits"] > 0
        _check(st, got, exp)
        ok, _, report = tree.validate()
        assert ok, report
    finally:
        tree.close()


def test_serve_rejects_bad_plans():
    import torch
    from indexingpu_b200.masstree import MasstreeError
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    st = wl.serve_stream(c2, 10, rate_per_s=1e4, disjoint=True)
    tree = _tree(torch, c2)
    try:
        bad = dict(st)
        bad["arrival_ns"] = st["arrival_ns"][::-1].copy()  # not in arrival order
        with pytest.raises(MasstreeError):
            _serve(torch, tree, bad)
        overlap = dict(st)
        overlap["first"] = st["first"].copy()
        overlap["first"][1] = st["first"][0]  # request 1 reuses request 0's ops
        with pytest.raises(MasstreeError):
            _serve(torch, tree, overlap)
        # The tree is still usable.
        _serve(torch, tree, st)
    finally:
        tree.close()
