"""Erase with MT_FLAG_MERGE (the reference's erase merge levels 2-4): sparse
border nodes, and then sparse interior nodes, are folded into a neighbour after
the call's erases, and a layer root left with one child takes it in.  Results
and the full ordered contents must equal the oracle's and the tree must
validate (sibling links included), through later inserts, finds and mixed
batches too; the merged tree must hold fewer slabs than the same tree erased
without merges."""
import numpy as np
import pytest

from indexes import GpuIndex, OracleIndex, same_state
from indexingpu_b200 import workload as wl
from scenarios import assert_found

pytestmark = pytest.mark.gpu


def _used(g):
    return g.t.stats()["used_slabs"]


@pytest.mark.parametrize("bulk", [True, False])
@pytest.mark.parametrize("write_tile", [8, 32])
def test_merge_after_erase_c1(bulk, write_tile):
    """C1 keys: 80% erased in two calls, with and without merges; then the
    erased keys inserted again."""
    n = 200000
    d = wl.c1(n_keys=n, n_finds=1000)
    keys, lens, vals, vlens = d["keys"], d["lens"], d["vals"], d["vlens"]
    gm, g0, o = GpuIndex(tile_size=8, pool_bytes=1 << 30), GpuIndex(tile_size=8, pool_bytes=1 << 30), OracleIndex()
    try:
        for g in (gm, g0):
            g.t.set_write_tile_size(write_tile)
            # One call takes the bulk build (packed nodes); chunks below its
            # minimum grow the tree by splits (half-full nodes).
            step = n if bulk else 40000
            for a in range(0, n, step):
                g.insert(keys[a:a + step], lens[a:a + step], vals[a:a + step], vlens[a:a + step])
        o.insert(keys, lens, vals, vlens)
        rng = np.random.default_rng(5)
        gone = rng.permutation(n)[: n * 8 // 10]
        for part in np.array_split(gone, 2):
            rm = gm.erase(keys[part], lens[part], merge=True)
            r0 = g0.erase(keys[part], lens[part])
            ro = o.erase(keys[part], lens[part])
            np.testing.assert_array_equal(rm, ro)
            np.testing.assert_array_equal(r0, ro)
        for g in (gm, g0):
            ok, nkeys, report = g.t.validate()
            assert ok, report
            assert nkeys == n - len(gone)
        same_state(gm, o, 8, 2)
        assert _used(gm) < 0.9 * _used(g0), (_used(gm), _used(g0))
        # Finds of everything, then the erased keys back in.
        gv, gl = gm.find(keys, lens, 2)
        ov, ol = o.find(keys, lens, 2)
        assert_found(gv, gl, ov, ol, "finds on the merged tree")
        np.testing.assert_array_equal(gm.insert(keys[gone], lens[gone], vals[gone], vlens[gone]),
                                      o.insert(keys[gone], lens[gone], vals[gone], vlens[gone]))
        ok, nkeys, report = gm.t.validate()
        assert ok, report
        assert nkeys == n
        same_state(gm, o, 8, 2)
    finally:
        gm.close()
        g0.close()


def test_merge_in_mixed_batches_c2():
    """C2 keys (shared prefixes, several trie layers): touch-once mixed batches
    that erase most of the tree with merges on, plus finds and inserts."""
    c2 = wl.C2(n_preload=120000, n_prefixes=64)
    keys, lens, vals, vlens = c2.keys(np.arange(120000))
    g, o = GpuIndex(tile_size=8, pool_bytes=1 << 30), OracleIndex()
    try:
        g.insert(keys, lens, vals, vlens)
        o.insert(keys, lens, vals, vlens)
        rng = np.random.default_rng(9)
        order = rng.permutation(120000)
        fresh = 120000
        for b in range(3):
            # 30,000 present keys per batch: 80% erased, 20% found; plus 2,000
            # new keys inserted.
            pick = order[b * 30000:(b + 1) * 30000]
            types = np.where(rng.random(30000) < 0.8, wl.REQ_ERASE, wl.REQ_FIND).astype(np.uint8)
            nk, nl, nv, nvl = c2.keys(np.arange(fresh, fresh + 2000))
            fresh += 2000
            types = np.concatenate([types, np.full(2000, wl.REQ_INSERT, np.uint8)])
            k = np.concatenate([keys[pick], nk])
            ln = np.concatenate([lens[pick], nl])
            v = np.concatenate([vals[pick], nv])
            vl = np.concatenate([np.where(types[:30000] == wl.REQ_FIND, 0, vlens[pick]), nvl]).astype(np.uint32)
            gv, gl, gr = g.mixed(types, k, ln, v, vl, merge=True)
            ov, ol, orr = o.mixed(types, k, ln, v, vl)
            nf = types != wl.REQ_FIND
            np.testing.assert_array_equal(gr[nf], orr[nf])
            assert_found(gv[~nf], gl[~nf], ov[~nf], ol[~nf], "mixed finds")
            ok, _, report = g.t.validate()
            assert ok, report
        same_state(g, o, c2.maxK, c2.maxV)
        # The rest erased through mt_erase with merges: layers emptied too.
        rest = order[90000:]
        np.testing.assert_array_equal(g.erase(keys[rest], lens[rest], merge=True), o.erase(keys[rest], lens[rest]))
        ok, nkeys, report = g.t.validate()
        assert ok, report
        assert nkeys == o.o.size()
        same_state(g, o, c2.maxK, c2.maxV)
    finally:
        g.close()


def _layered_keys(n_first, seed):
    """Keys of 2-4 slices under n_first distinct first slices A: [A,B], [A,B,C]
    and [A,B,C,D] for B in 3 values, C in 4, D in 2, so every A owns 16 trie
    layers of one border node each (its layer 1, three layers 2, twelve
    layers 3).  Values of 1-8 random slices."""
    rng = np.random.default_rng(seed)
    firsts = np.unique(rng.integers(0, 1 << 32, 2 * n_first, dtype=np.uint64).astype(np.uint32))[:n_first]
    rng.shuffle(firsts)
    rows = []
    for b in (5, 9, 1 << 31):
        rows.append([b, 0, 0, 2])
        for c in (0, 7, 1000, 0xFFFFFFFF):
            rows.append([b, c, 0, 3])
            for d in (3, 4):
                rows.append([b, c, d, 4])
    per = np.array(rows, dtype=np.uint32)  # 39 key shapes per first slice
    n = n_first * len(per)
    keys = np.zeros((n, 4), np.uint32)
    keys[:, 0] = np.repeat(firsts, len(per))
    keys[:, 1:] = np.tile(per[:, :3], (n_first, 1))
    lens = np.tile(per[:, 3], n_first).astype(np.uint32)
    keys[lens < 3, 2] = 0
    keys[lens < 4, 3] = 0
    vlens = rng.integers(1, 9, n).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, (n, 8), dtype=np.uint64).astype(np.uint32)
    vals[np.arange(8)[None, :] >= vlens[:, None]] = 0
    return firsts, keys, lens, vals, vlens


def test_remove_emptied_layers():
    """MT_FLAG_REMOVE_EMPTY_LAYERS (the reference's erase merge level 4): every
    key under half the first slices erased, half through mt_erase and half in a
    mixed batch beside finds, plus every key under one second slice of other
    first slices.  Results and contents equal the oracle's and the tree
    validates; it holds about 16 slabs fewer per emptied first slice than a
    tree erased with merges alone; the erased keys go back in; erasing
    everything then leaves only layer 0's nodes."""
    n_first = 1000
    firsts, keys, lens, vals, vlens = _layered_keys(n_first, 21)
    n = len(keys)
    gr, g0, o = GpuIndex(tile_size=8, pool_bytes=256 << 20), GpuIndex(tile_size=8, pool_bytes=256 << 20), OracleIndex()
    try:
        for g in (gr, g0, o):
            g.insert(keys, lens, vals, vlens)
        rng = np.random.default_rng(22)
        whole = np.isin(keys[:, 0], firsts[:500])
        part = np.isin(keys[:, 0], firsts[500:750]) & (keys[:, 1] == 9)
        gone = np.flatnonzero(whole | part)
        rng.shuffle(gone)
        a, b = gone[: len(gone) // 2], gone[len(gone) // 2:]
        ro = o.erase(keys[a], lens[a])
        np.testing.assert_array_equal(gr.erase(keys[a], lens[a], merge=True, remove_empty_layers=True), ro)
        np.testing.assert_array_equal(g0.erase(keys[a], lens[a], merge=True), ro)
        keep = rng.choice(np.flatnonzero(~(whole | part)), 5000, replace=False)
        idx = np.concatenate([b, keep])
        types = np.concatenate([np.full(len(b), wl.REQ_ERASE, np.uint8), np.full(len(keep), wl.REQ_FIND, np.uint8)])
        perm = rng.permutation(len(idx))
        idx, types = idx[perm], types[perm]
        vl = np.where(types == wl.REQ_FIND, 0, vlens[idx]).astype(np.uint32)
        ov, ol, orr = o.mixed(types, keys[idx], lens[idx], vals[idx], vl)
        gv, gl, grr = gr.mixed(types, keys[idx], lens[idx], vals[idx], vl, merge=True, remove_empty_layers=True)
        _, _, g0r = g0.mixed(types, keys[idx], lens[idx], vals[idx], vl, merge=True)
        nf = types != wl.REQ_FIND
        np.testing.assert_array_equal(grr[nf], orr[nf])
        np.testing.assert_array_equal(g0r[nf], orr[nf])
        assert_found(gv[~nf], gl[~nf], ov[~nf], ol[~nf], "finds beside the erases")
        for g in (gr, g0):
            ok, nkeys, report = g.t.validate()
            assert ok, report
            assert nkeys == n - len(gone)
        same_state(gr, o, 4, 8)
        # 16 layers per emptied first slice, 5 (one layer 2, four layers 3) per
        # emptied second slice; the two trees' layer 0 may differ by a few
        # nodes (concurrent inserts split at different moments).
        removed = 500 * 16 + 250 * 5
        assert _used(g0) - _used(gr) >= removed - 64, (_used(gr), _used(g0), removed)
        # The erased keys back in: their layers are built again.
        np.testing.assert_array_equal(gr.insert(keys[gone], lens[gone], vals[gone], vlens[gone]),
                                      o.insert(keys[gone], lens[gone], vals[gone], vlens[gone]))
        ok, nkeys, report = gr.t.validate()
        assert ok, report
        assert nkeys == n
        same_state(gr, o, 4, 8)
        gv, gl = gr.find(keys, lens, 8)
        ov, ol = o.find(keys, lens, 8)
        assert_found(gv, gl, ov, ol, "finds after the keys went back in")
        # Everything erased: no layer below layer 0 is left.
        full = _used(gr)
        np.testing.assert_array_equal(gr.erase(keys, lens, merge=True, remove_empty_layers=True),
                                      o.erase(keys, lens))
        ok, nkeys, report = gr.t.validate()
        assert ok, report
        assert nkeys == 0
        # Layer 0 lost its LINK entries in the removal pass; merged upwards,
        # it folded back into its root.
        assert _used(gr) == 1, (_used(gr), full)
        same_state(gr, o, 4, 8)
    finally:
        gr.close()
        g0.close()


def _one_layer_keys(n, seed):
    """n distinct one-slice keys with one-slice values (every entry inline in
    layer 0)."""
    rng = np.random.default_rng(seed)
    s = np.unique(rng.integers(0, 1 << 32, 2 * n, dtype=np.uint64).astype(np.uint32))[:n]
    rng.shuffle(s)
    keys = s.reshape(n, 1).copy()
    vals = rng.integers(0, 1 << 32, (n, 1), dtype=np.uint64).astype(np.uint32)
    return keys, np.ones(n, np.uint32), vals, np.ones(n, np.uint32)


@pytest.mark.parametrize("write_tile", [8, 32])
def test_interior_merges_and_root_collapse(write_tile):
    """300,000 one-slice keys grown by splits (a layer of six levels), 96%
    erased in three calls: interior nodes merge as well as border nodes, so
    the merged tree holds few more slabs than a tree built from the surviving
    keys alone.  Erasing the rest folds the layer back into its root slab (one
    slab in use); the keys then go back in."""
    n = 300000
    keys, lens, vals, vlens = _one_layer_keys(n, 31)
    gm, g0, gf, o = (GpuIndex(tile_size=8, pool_bytes=256 << 20), GpuIndex(tile_size=8, pool_bytes=256 << 20),
                     GpuIndex(tile_size=8, pool_bytes=256 << 20), OracleIndex())
    try:
        for g in (gm, g0):
            g.t.set_write_tile_size(write_tile)
            for a in range(0, n, 30000):
                g.insert(keys[a:a + 30000], lens[a:a + 30000], vals[a:a + 30000], vlens[a:a + 30000])
        o.insert(keys, lens, vals, vlens)
        rng = np.random.default_rng(32)
        perm = rng.permutation(n)
        gone, kept = perm[: n * 96 // 100], perm[n * 96 // 100:]
        for part in np.array_split(gone, 3):
            ro = o.erase(keys[part], lens[part])
            np.testing.assert_array_equal(gm.erase(keys[part], lens[part], merge=True), ro)
            np.testing.assert_array_equal(g0.erase(keys[part], lens[part]), ro)
            ok, nkeys, report = gm.t.validate()
            assert ok, report
        gf.insert(keys[kept], lens[kept], vals[kept], vlens[kept])
        assert nkeys == len(kept)
        same_state(gm, o, 1, 1)
        used_m, used_0, used_f = _used(gm), _used(g0), _used(gf)
        print(f"slabs after 96% erased: merged {used_m}, unmerged {used_0}, built from the rest {used_f}")
        assert used_m < 2 * used_f, (used_m, used_f)
        gv, gl = gm.find(keys, lens, 1)
        ov, ol = o.find(keys, lens, 1)
        assert_found(gv, gl, ov, ol, "finds on the merged tree")
        # Everything else erased (with a mixed batch of finds beside): one slab.
        types = np.concatenate([np.full(len(kept), wl.REQ_ERASE, np.uint8), np.full(1000, wl.REQ_FIND, np.uint8)])
        idx = np.concatenate([kept, gone[:1000]])
        sh = rng.permutation(len(idx))
        types, idx = types[sh], idx[sh]
        vl = np.where(types == wl.REQ_FIND, 0, 1).astype(np.uint32)
        gv, gl, gr = gm.mixed(types, keys[idx], lens[idx], vals[idx], vl, merge=True)
        ov, ol, orr = o.mixed(types, keys[idx], lens[idx], vals[idx], vl)
        nf = types != wl.REQ_FIND
        np.testing.assert_array_equal(gr[nf], orr[nf])
        assert_found(gv[~nf], gl[~nf], ov[~nf], ol[~nf], "finds beside the last erases")
        ok, nkeys, report = gm.t.validate()
        assert ok, report
        assert nkeys == 0
        assert _used(gm) == 1, _used(gm)
        np.testing.assert_array_equal(gm.insert(keys, lens, vals, vlens), o.insert(keys, lens, vals, vlens))
        ok, nkeys, report = gm.t.validate()
        assert ok, report
        assert nkeys == n
        same_state(gm, o, 1, 1)
    finally:
        gm.close()
        g0.close()
        gf.close()
