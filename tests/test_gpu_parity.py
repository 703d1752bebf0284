"""Parity of the CUDA library with the CPU oracle on seeded workloads shaped
like the benchmark configurations, at sizes the oracle finishes in seconds.
Integer results must match bit-for-bit.
"""
import numpy as np
import pytest

from indexes import GpuIndex, OracleIndex, same_state
from indexingpu_b200 import workload as wl
from scenarios import assert_found

pytestmark = pytest.mark.gpu
TILES = [4, 8, 16, 32]


@pytest.fixture(params=TILES)
def tile(request):
    return request.param


def dump_via_scan(idx, maxK, maxV, n_expected):
    """Every key in order, by one scan from the smallest possible key."""
    lower = np.zeros((1, maxK), np.uint32)
    counts, vals, vlens, okeys, oklens = idx.scan(lower, np.ones(1, np.uint32), n_expected + 8, maxV=maxV)
    c = int(counts[0])
    return okeys[0, :c], oklens[0, :c], vals[0, :c], vlens[0, :c]


def assert_same_state(a, b, what):
    ka, la, va, vla = a
    kb, lb, vb, vlb = b
    assert len(la) == len(lb), f"{what}: {len(la)} vs {len(lb)} keys"
    np.testing.assert_array_equal(la, lb, err_msg=f"{what}: key lengths")
    np.testing.assert_array_equal(vla, vlb, err_msg=f"{what}: value lengths")
    for i in range(len(la)):
        L = la[i]
        assert np.array_equal(ka[i, :L], kb[i, :L]), f"{what}: key {i}"
        c = min(int(vla[i]), va.shape[1])
        assert np.array_equal(va[i, :c], vb[i, :c]), f"{what}: value {i}"


def test_c1_insert_find(tile):
    w = wl.c1(n_keys=20000, n_finds=20000)
    g, o = GpuIndex(tile), OracleIndex()
    try:
        rg = g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        ro = o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        np.testing.assert_array_equal(rg, ro)
        assert rg.all()
        for conc in (False, True):
            vg, lg = g.find(w["find_keys"], w["find_lens"], 2, concurrent=conc)
            vo, lo = o.find(w["find_keys"], w["find_lens"], 2)
            assert_found(vg, lg, vo, lo, f"c1 find concurrent={conc}")
            assert (lg > 0).sum() == w["find_hit"].sum()
    finally:
        g.close()


def test_find_value_truncation_and_null_lengths(tile):
    # Stored values longer than max_value_length: the full length is returned
    # and max_value_length slices are written.
    keys = np.arange(1, 301, dtype=np.uint32).reshape(100, 3)
    lens = np.full(100, 3, np.uint32)
    vals = np.tile(np.arange(7, dtype=np.uint32), (100, 1)) + keys[:, :1]
    vlens = np.full(100, 7, np.uint32)
    g = GpuIndex(tile)
    try:
        g.insert(keys, lens, vals, vlens)
        v, l = g.find(keys, None, 3)  # NULL key lengths -> every key has max length 3
        assert (l == 7).all()
        np.testing.assert_array_equal(v, vals[:, :3])
    finally:
        g.close()


def test_upsert_and_results(tile):
    w = wl.c1(n_keys=5000, n_finds=10)
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        v2 = w["vals"] ^ np.uint32(0x5A5A5A5A)
        # Mixed 1-slice and 2-slice new values: VALUE <-> LONGVAL transitions.
        vl2 = (1 + (np.arange(len(v2)) % 2)).astype(np.uint32)
        np.testing.assert_array_equal(g.insert(w["keys"], w["lens"], v2, vl2, upsert=True),
                                      o.insert(w["keys"], w["lens"], v2, vl2, upsert=True))
        vg, lg = g.find(w["keys"], w["lens"], 2)
        vo, lo = o.find(w["keys"], w["lens"], 2)
        assert_found(vg, lg, vo, lo, "upsert")
        # Plain insert of existing keys fails everywhere.
        assert not g.insert(w["keys"], w["lens"], v2, vl2).any()
    finally:
        g.close()


def _touch_once_batches(c2, n_batches, n):
    """Mixed batches in which every key appears at most once (per-request
    results are order independent)."""
    out = []
    for b in range(n_batches):
        bt = c2.batch(b, n)
        _, first = np.unique(bt["ids"], return_index=True)
        keep = np.sort(first)
        out.append({k: v[keep] for k, v in bt.items()})
    return out


@pytest.mark.parametrize("bucket", [False, True])
@pytest.mark.parametrize("n_preload", [3000, 40000])
def test_c2_mixed_touch_once(tile, n_preload, bucket):
    c2 = wl.C2(n_preload=n_preload, n_prefixes=64)
    keys, lens, vals, vlens = c2.keys(np.arange(n_preload))
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(keys, lens, vals, vlens)
        o.insert(keys, lens, vals, vlens)
        for bt in _touch_once_batches(c2, 4, 8000):
            gv, gl, gr = g.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"], bucket_keys=bucket)
            ov, ol, orr = o.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
            notfind = bt["types"] != wl.REQ_FIND
            np.testing.assert_array_equal(gr[notfind], orr[notfind], err_msg="mixed results")
            f = ~notfind
            assert_found(gv[f], gl[f], ov[f], ol[f], "mixed finds")
        assert_same_state(dump_via_scan(g, 16, 8, o.o.size()), o.dump(16, 8), "final state")
    finally:
        g.close()


def test_c2_mixed_zipf_final_state(tile):
    """Zipf batches with repeated keys: final key set and values are
    deterministic (fresh inserts, key-determined update values, erase wins)."""
    c2 = wl.C2(n_preload=20000, n_prefixes=64)
    keys, lens, vals, vlens = c2.keys(np.arange(20000))
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(keys, lens, vals, vlens)
        o.insert(keys, lens, vals, vlens)
        for b in range(3):
            bt = c2.batch(b, 20000)
            # Deterministic final state: updates of a key that the batch also
            # erases are dropped from both sides' final comparison by erasing
            # last; run updates only on keys not erased in this batch.
            er = set(bt["ids"][bt["types"] == wl.REQ_ERASE].tolist())
            keep = np.array([not (t == wl.REQ_UPDATE and i in er) for t, i in zip(bt["types"], bt["ids"])])
            bt = {k: v[keep] for k, v in bt.items()}
            g.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
            o.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
        assert_same_state(dump_via_scan(g, 16, 8, o.o.size()), o.dump(16, 8), "final state")
    finally:
        g.close()


def test_c3_scan(tile):
    w = wl.c3(50000, 3000)
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        rg = g.scan(w["lower"], w["lower_lens"], 100, maxV=1)
        ro = o.scan(w["lower"], w["lower_lens"], 100, maxV=1)
        for a, b, name in zip(rg, ro, ["counts", "values", "value_lengths", "keys", "key_lengths"]):
            np.testing.assert_array_equal(a, b, err_msg=f"scan {name}")
    finally:
        g.close()


@pytest.mark.parametrize("scan_tile", [4, 32])
def test_c3_scan_own_tile_width(scan_tile):
    """Scans with their own tile width (mt_set_scan_tile_size) beside finds of
    another: identical results to the oracle."""
    w = wl.c3(50000, 3000)
    g, o = GpuIndex(8), OracleIndex()
    try:
        g.t.set_scan_tile_size(scan_tile)
        g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        rg = g.scan(w["lower"], w["lower_lens"], 100, maxV=1)
        ro = o.scan(w["lower"], w["lower_lens"], 100, maxV=1)
        for a, b, name in zip(rg, ro, ["counts", "values", "value_lengths", "keys", "key_lengths"]):
            np.testing.assert_array_equal(a, b, err_msg=f"scan {name}")
        gv, gl = g.find(w["keys"][:5000], w["lens"][:5000], 1)
        np.testing.assert_array_equal(gl, np.ones(5000, np.uint32))
    finally:
        g.close()


def test_scan_with_upper_varlen(tile):
    c2 = wl.C2(n_preload=30000, n_prefixes=16)
    keys, lens, vals, vlens = c2.keys(np.arange(30000))
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(keys, lens, vals, vlens)
        o.insert(keys, lens, vals, vlens)
        rng = np.random.default_rng(5)
        a = rng.integers(0, 30000, 2000)
        b = rng.integers(0, 30000, 2000)
        lo_k, lo_l = keys[a].copy(), lens[a].copy()
        up_k, up_l = keys[b].copy(), lens[b].copy()
        # Some bounds are shortened prefixes of stored keys (absent keys).
        cut = rng.random(2000) < 0.3
        lo_l = np.where(cut, np.maximum(1, lo_l - 1), lo_l)
        for mc in (7, 50):
            rg = g.scan(lo_k, lo_l, mc, up_k, up_l, maxV=8)
            ro = o.scan(lo_k, lo_l, mc, up_k, up_l, maxV=8)
            np.testing.assert_array_equal(rg[0], ro[0], err_msg="counts")
            for q in range(2000):
                c = int(ro[0][q])
                np.testing.assert_array_equal(rg[4][q, :c], ro[4][q, :c])
                np.testing.assert_array_equal(rg[2][q, :c], ro[2][q, :c])
                for r in range(c):
                    L = ro[4][q, r]
                    assert np.array_equal(rg[3][q, r, :L], ro[3][q, r, :L])
                    V = min(int(ro[2][q, r]), 8)
                    assert np.array_equal(rg[1][q, r, :V], ro[1][q, r, :V])
    finally:
        g.close()


def test_empty_batches_and_pool_exhaustion():
    g = GpuIndex(8, pool_bytes=64 * 136 * 64)  # 4096 slabs
    try:
        # Zero-sized calls are no-ops.
        z = np.zeros((0, 4), np.uint32)
        g.t.insert(None, 4, None, None, 1, None, 0)
        w = wl.c1(n_keys=20000, n_finds=10)
        from indexingpu_b200 import MasstreeError
        with pytest.raises(MasstreeError) as e:
            g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        assert e.value.code == 1  # MT_ERR_OOM, reported, no hang
        del z
    finally:
        g.close()


@pytest.mark.parametrize("depth", [40, 300])
def test_scan_layers_beyond_scratch(tile, depth):
    # Keys sharing `depth` - 2 leading slices build that many one-entry trie
    # layers (suffix splits), so a scan descends deeper than the 32 layer
    # frames held in scratch and spills the rest to slabs.
    rng = np.random.default_rng(depth)
    n = 24
    maxK = depth + 1
    keys = np.zeros((n, maxK), np.uint32)
    keys[:, : depth - 2] = rng.integers(1, 1 << 32, depth - 2, dtype=np.uint32)
    keys[:, depth - 2:] = rng.integers(0, 1 << 32, (n, 3), dtype=np.uint32)
    lens = np.full(n, depth, np.uint32)
    lens[::3] = depth + 1
    vals = rng.integers(0, 1 << 32, (n, 2), dtype=np.uint32)
    vlens = np.full(n, 2, np.uint32)
    g, o = GpuIndex(tile), OracleIndex()
    try:
        np.testing.assert_array_equal(g.insert(keys, lens, vals, vlens), o.insert(keys, lens, vals, vlens))
        lower = np.zeros((3, maxK), np.uint32)
        lower[1] = keys[5]
        lower[2, : depth - 2] = keys[0, : depth - 2]
        llen = np.array([1, lens[5], depth - 2], np.uint32)
        a = g.scan(lower, llen, n + 4, maxV=2)
        b = o.scan(lower, llen, n + 4, maxV=2)
        for x, y, name in zip(a, b, ["counts", "values", "value lengths", "keys", "key lengths"]):
            np.testing.assert_array_equal(x, y, err_msg=name)
        assert a[0][0] == n
        g.t.reclaim()
        st = g.t.stats()
        assert st["limbo_slabs"] == 0 and st["device_error"] == 0
    finally:
        g.close()


def test_combined_updates_of_hot_keys(tile):
    # Many updates of few keys in one call (what skewed key choice gives): all
    # but one per key are combined into the one that runs and report its
    # result.  Keys present and not erased in the call: every update true;
    # absent keys: every update false; the final contents are the oracle's
    # (the update values of one key are equal, as in the benchmark streams).
    c2 = wl.C2(n_preload=5000, n_prefixes=64)
    k, l, v, vl = c2.keys(np.arange(5000))
    g, o = GpuIndex(tile), OracleIndex()
    try:
        g.insert(k, l, v, vl)
        o.insert(k, l, v, vl)
        rng = np.random.default_rng(tile)
        hot = rng.choice(3000, 40, replace=False)  # none of the keys erased below
        absent_k, absent_l, _, _ = c2.keys(np.arange(6000, 6010))
        ids = np.concatenate([np.repeat(hot, 300), np.arange(3000, 3200)])
        uk = np.concatenate([k[ids], np.repeat(absent_k, 50, axis=0)])
        ul = np.concatenate([l[ids], np.repeat(absent_l, 50)])
        uv = np.concatenate([v[ids] ^ np.uint32(0x77), np.zeros((500, 8), np.uint32)])
        uvl = np.concatenate([vl[ids], np.full(500, 3, np.uint32)])
        perm = rng.permutation(len(uk))
        uk, ul, uv, uvl = uk[perm], ul[perm], uv[perm], uvl[perm]
        rg = g.update(uk, ul, uv, uvl)
        ro = o.update(uk, ul, uv, uvl)
        np.testing.assert_array_equal(rg, ro)  # present: true, absent: false, whatever the order
        same_state(g, o, 16, 8)
        # The same inside mixed batches, with finds of the hot keys, and erases
        # of other keys' duplicates (their updates may go either way).
        types = np.full(len(uk), wl.REQ_UPDATE, np.uint8)
        fk = k[hot]
        erase_ids = np.arange(3200, 3260)
        bk = np.concatenate([uk, fk, k[erase_ids], k[erase_ids]])
        bl = np.concatenate([ul, l[hot], l[erase_ids], l[erase_ids]])
        bv = np.concatenate([uv ^ np.uint32(1), np.zeros((len(hot) + 120, 8), np.uint32)])
        bvl = np.concatenate([uvl, np.zeros(len(hot) + 120, np.uint32)])
        bt = np.concatenate([types, np.full(len(hot), wl.REQ_FIND, np.uint8), np.full(60, wl.REQ_ERASE, np.uint8),
                             np.full(60, wl.REQ_UPDATE, np.uint8)])
        bv[-60:] = 5
        bvl[-60:] = 2
        gv, gl, gr = g.mixed(bt, bk, bl, bv, bvl)
        o.mixed(bt, bk, bl, bv, bvl)
        n_upd = len(uk)
        np.testing.assert_array_equal(gr[:n_upd], rg)  # the hot keys stay present: same results as before
        assert (gl[n_upd:n_upd + len(hot)] > 0).all()
        same_state(g, o, 16, 8)
        ok, nkeys, msg = g.t.validate()
        assert ok and nkeys == o.o.size(), msg
    finally:
        g.close()
