"""mt_mixed_batches (many sub-batches in one persistent launch) against one
mt_mixed_batch call per sub-batch on an identical tree: per-request results,
find outputs and the final contents must match exactly; with and without key
bucketing, every find tile width, and replayed from a captured CUDA graph."""
import numpy as np
import pytest

from indexingpu_b200 import workload as wl
from indexingpu_b200.masstree import pack_subbatches

pytestmark = pytest.mark.gpu
MAXK, MAXV = 16, 8


def _touch_once(bt):
    _, first = np.unique(bt["ids"], return_index=True)
    keep = np.sort(first)
    return {k: v[keep] for k, v in bt.items()}


def _dev(torch, bt):
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in bt.items() if k != "ids"}
    n = len(bt["types"])
    return dict(types=d["types"], keys=d["keys"], lens=d["lens"], vals=d["vals"].clone(), vlens=d["vlens"].clone(),
                results=torch.zeros(n, dtype=torch.bool, device="cuda"), n=n)


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


def _make_pair(torch, c2, n_pre, tf, tw):
    from indexingpu_b200 import GpuMasstree
    keys, lens, vals, vlens = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c2.keys(np.arange(n_pre)))
    trees = []
    for _ in range(2):
        t = GpuMasstree(pool_bytes=512 << 20, tile_size=tf)
        t.set_write_tile_size(tw)
        t.insert(keys, MAXK, lens, vals, MAXV, vlens, n_pre)
        t.sync()
        trees.append(t)
    return trees


def _compare(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def _check_outputs(ref_sb, new_sb, bt):
    types = bt["types"]
    find = types == wl.REQ_FIND
    np.testing.assert_array_equal(new_sb["results"].cpu().numpy()[~find], ref_sb["results"].cpu().numpy()[~find])
    gl, el = new_sb["vlens"].cpu().numpy(), ref_sb["vlens"].cpu().numpy()
    np.testing.assert_array_equal(gl[find], el[find])
    gv, ev = new_sb["vals"].cpu().numpy(), ref_sb["vals"].cpu().numpy()
    for i in np.nonzero(find & (el > 0))[0]:
        c = min(int(el[i]), MAXV)
        assert np.array_equal(gv[i, :c], ev[i, :c]), i


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("tf,tw,bucket", [(8, 32, False), (8, 32, True), (4, 16, True), (16, 32, False),
                                          (32, 32, True)])
def test_mixed_batches_match_per_call(tf, tw, bucket, persistent):
    import torch
    c2 = wl.C2(n_preload=20000, n_prefixes=64)
    ref, new = _make_pair(torch, c2, 20000, tf, tw)
    try:
        sizes = [3000, 17, 900, 5000, 1, 2500, 128, 4096]
        bts = [_touch_once(c2.batch(b, n)) for b, n in enumerate(sizes)]
        ref_sbs = [_dev(torch, bt) for bt in bts]
        new_sbs = [_dev(torch, bt) for bt in bts]
        for sb in ref_sbs:
            ref.mixed_batch(sb["types"], sb["keys"], MAXK, sb["lens"], sb["vals"], MAXV, sb["vlens"], sb["results"],
                            sb["n"])
        ref.sync()
        desc = torch.from_numpy(pack_subbatches(new_sbs)).cuda()
        new.reserve_batches(len(new_sbs), sum(sb["n"] for sb in new_sbs))
        new.mixed_batches(desc, len(new_sbs), MAXK, MAXV, bucket_keys=bucket, persistent=persistent)
        new.sync()
        for r, s, bt in zip(ref_sbs, new_sbs, bts):
            _check_outputs(r, s, bt)
        _compare(_dump(torch, ref, 60000), _dump(torch, new, 60000))
        ok, _, msg = new.validate()
        assert ok, msg
    finally:
        ref.close()
        new.close()


@pytest.mark.parametrize("form", ["forked", "persistent", "grouped"])
def test_mixed_batches_graph_replay(form):
    """Capture one mt_mixed_batches call in a CUDA graph, then replay it after
    rewriting the sub-batch buffers in place with the next batches' data (the
    grouped form's scratch is sized by its first call, before the capture)."""
    persistent, grouped = form == "persistent", form == "grouped"
    import torch
    c2 = wl.C2(n_preload=20000, n_prefixes=64)
    ref, new = _make_pair(torch, c2, 20000, 8, 32)
    try:
        sizes = [2000, 700, 3000]
        rounds = 3
        plans = [[_touch_once(c2.batch(10 * r + b, n)) for b, n in enumerate(sizes)] for r in range(rounds)]
        cap = max(len(bt["types"]) for p in plans for bt in p)
        # Fixed buffers the graph points at.
        bufs = [dict(types=torch.zeros(cap, dtype=torch.uint8, device="cuda"),
                     keys=torch.zeros((cap, MAXK), dtype=torch.uint32, device="cuda"),
                     lens=torch.zeros(cap, dtype=torch.uint32, device="cuda"),
                     vals=torch.zeros((cap, MAXV), dtype=torch.uint32, device="cuda"),
                     vlens=torch.zeros(cap, dtype=torch.uint32, device="cuda"),
                     results=torch.zeros(cap, dtype=torch.bool, device="cuda"), n=cap) for _ in sizes]
        desc = torch.from_numpy(pack_subbatches(bufs)).cuda()
        new.reserve_batches(len(bufs), cap * len(bufs))

        def load(plan):
            # Same sizes every round: pad each sub-batch to cap with finds of key 0.
            for buf, bt in zip(bufs, plan):
                n = len(bt["types"])
                t = np.full(cap, wl.REQ_FIND, np.uint8)
                t[:n] = bt["types"]
                buf["types"].copy_(torch.from_numpy(t))
                k = np.zeros((cap, MAXK), np.uint32)
                k[:n] = bt["keys"]
                buf["keys"].copy_(torch.from_numpy(k))
                ln = np.ones(cap, np.uint32)
                ln[:n] = bt["lens"]
                buf["lens"].copy_(torch.from_numpy(ln))
                v = np.zeros((cap, MAXV), np.uint32)
                v[:n] = bt["vals"]
                buf["vals"].copy_(torch.from_numpy(v))
                vl = np.zeros(cap, np.uint32)
                vl[:n] = bt["vlens"]
                buf["vlens"].copy_(torch.from_numpy(vl))
            torch.cuda.synchronize()

        # Warm-up call outside capture (first-call setup), on the first plan's data.
        load(plans[0])
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            new.mixed_batches(desc, len(bufs), MAXK, MAXV, stream=s, persistent=persistent, group_by_key=grouped)
        new.sync(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            new.mixed_batches(desc, len(bufs), MAXK, MAXV, stream=s, persistent=persistent, group_by_key=grouped)
        for r in range(1, rounds):
            load(plans[r])
            g.replay()
            new.sync(s)
        # Reference: the same padded sub-batches, one call each, in the same order.
        for r in range(rounds):
            load(plans[r])
            for buf in bufs:
                ref.mixed_batch(buf["types"], buf["keys"], MAXK, buf["lens"], buf["vals"], MAXV, buf["vlens"],
                                buf["results"], cap)
            ref.sync()
        _compare(_dump(torch, ref, 60000), _dump(torch, new, 60000))
        del g
    finally:
        ref.close()
        new.close()


def test_autotune_small_cases():
    """The autotuner runs every trial through mt_mixed_batches on fresh cases,
    returns a configuration from its grid, and leaves a valid tree."""
    import torch
    from indexingpu_b200 import GpuMasstree, autotune
    c2 = wl.C2(n_preload=20000, n_prefixes=64)
    keys, lens, vals, vlens = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c2.keys(np.arange(20000)))
    t = GpuMasstree(pool_bytes=512 << 20, tile_size=8)
    try:
        t.insert(keys, MAXK, lens, vals, MAXV, vlens, 20000)
        t.sync()

        def make_case(i):
            st = wl.serve_stream(c2, 4, min_ops=64, max_ops=4096, seed=11, op_seed=100 + i,
                                 first_fresh=(1 << 20) + i * (1 << 16))
            d = {k: torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in ("types", "keys", "lens", "vals",
                                                                                    "vlens")}
            res = torch.zeros(len(st["types"]), dtype=torch.bool, device="cuda")
            subs = []
            for f, n in zip(st["first"].tolist(), st["nops"].tolist()):
                subs.append(dict(types=d["types"][f:f + n], keys=d["keys"][f:f + n], lens=d["lens"][f:f + n],
                                 vals=d["vals"][f:f + n], vlens=d["vlens"][f:f + n], results=res[f:f + n], n=n))
            desc = torch.from_numpy(pack_subbatches(subs)).cuda()
            return dict(descriptors=desc, num_subbatches=len(subs), total=int(st["nops"].sum()),
                        max_key_length=MAXK, max_value_length=MAXV, keep=(d, res))

        best, trials = autotune.tune(t, make_case, blocks_per_sm=(2, 8))
        assert len(trials) == 2 * 16 + 8 + 2  # forked and persistent x 16 shapes, grouped x 8, blocks per SM x 2
        assert best["form"] in autotune.FORMS
        assert best["find_tile"] in autotune.FIND_TILES and best["write_tile"] in autotune.WRITE_TILES
        assert all(tr["mops"] > 0 for tr in trials)
        ok, _, report = t.validate()
        assert ok, report
    finally:
        t.close()
