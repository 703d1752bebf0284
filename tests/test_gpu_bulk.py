"""An insert of 1,024 keys or more into an empty tree bulk-builds its first
layer: one entry per key alone at its first slice, a LINK entry to a new layer
for keys that continue past a shared first slice (those keys are then inserted
below it).  Results, found values and the full ordered contents must equal the
oracle's, the tree must validate, and it must keep working under ordinary
mixed batches."""
import numpy as np
import pytest

from indexes import GpuIndex, OracleIndex, same_state
from indexingpu_b200 import workload as wl
from scenarios import assert_found

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tile", [8, 32])
def test_bulk_build_c1(tile):
    d = wl.c1(n_keys=200000, n_finds=100000)
    g, o = GpuIndex(tile_size=tile, pool_bytes=1 << 30), OracleIndex()
    try:
        gr = g.insert(d["keys"], d["lens"], d["vals"], d["vlens"])
        orr = o.insert(d["keys"], d["lens"], d["vals"], d["vlens"])
        np.testing.assert_array_equal(gr, orr)
        assert gr.all()
        gv, gl = g.find(d["find_keys"], d["find_lens"], 2)
        ov, ol = o.find(d["find_keys"], d["find_lens"], 2)
        assert_found(gv, gl, ov, ol, "finds after a bulk build")
        assert int((gl > 0).sum()) == int(d["find_hit"].sum())
        ok, nkeys, report = g.t.validate()
        assert ok, report
        assert nkeys == 200000
        same_state(g, o, 8, 2)
    finally:
        g.close()


@pytest.mark.parametrize("upsert", [False, True])
def test_bulk_build_duplicates_and_shared_slices(upsert):
    """A batch where keys repeat (same value) and share first slices with
    other keys: the shared ones go through the ordinary insert."""
    rng = np.random.default_rng(7)
    n = 120000
    maxK, maxV = 6, 3
    lens = rng.integers(1, maxK + 1, n).astype(np.uint32)
    keys = rng.integers(0, 1 << 32, (n, maxK), dtype=np.uint64).astype(np.uint32)
    keys[np.arange(maxK)[None, :] >= lens[:, None]] = 0
    # 30% share their first slice with an earlier key, 10% repeat an earlier key.
    share = rng.random(n) < 0.3
    src = rng.integers(0, n // 2, n)
    keys[share, 0] = keys[src[share], 0]
    dup = rng.random(n) < 0.1
    dup_src = rng.integers(0, n // 2, n)
    keys[dup] = keys[dup_src[dup]]
    lens[dup] = lens[dup_src[dup]]
    vlens = rng.integers(1, maxV + 1, n).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, (n, maxV), dtype=np.uint64).astype(np.uint32)
    # One-slice keys that took another's first slice are copies too: every
    # copy of a key carries its first occurrence's value, so which copy
    # lands is not observable.
    _, first, inv = np.unique(np.column_stack([keys, lens]), axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    vals, vlens = vals[first[inv]], vlens[first[inv]]
    g, o = GpuIndex(tile_size=8, pool_bytes=1 << 30), OracleIndex()
    try:
        gr = g.insert(keys, lens, vals, vlens, upsert=upsert)
        orr = o.insert(keys, lens, vals, vlens, upsert=upsert)
        # Repeated keys: which copy reports the insert is not defined, the
        # number of reported inserts (or updates) is.
        assert int(gr.sum()) == int(orr.sum())
        ok, nkeys, report = g.t.validate()
        assert ok, report
        same_state(g, o, maxK, maxV)
    finally:
        g.close()


def test_bulk_built_tree_takes_mixed_batches():
    d = wl.c1(n_keys=150000, n_finds=1000)
    g, o = GpuIndex(tile_size=8, pool_bytes=1 << 30), OracleIndex()
    try:
        g.insert(d["keys"], d["lens"], d["vals"], d["vlens"])
        o.insert(d["keys"], d["lens"], d["vals"], d["vlens"])
        rng = np.random.default_rng(3)
        for b in range(3):
            # Touch-once batch: erases and updates of present keys, finds,
            # inserts of new keys (from the finds' absent half).
            pick = rng.choice(150000, 20000, replace=False)
            types = rng.choice([wl.REQ_FIND, wl.REQ_UPDATE, wl.REQ_ERASE], 20000).astype(np.uint8)
            k, ln = d["keys"][pick], d["lens"][pick]
            v = rng.integers(0, 1 << 32, (20000, 2), dtype=np.uint64).astype(np.uint32)
            vl = np.where(types == wl.REQ_FIND, 0, 2).astype(np.uint32)
            miss = ~d["find_hit"]
            nk = d["find_keys"][miss][b * 100:(b + 1) * 100]
            nl = d["find_lens"][miss][b * 100:(b + 1) * 100]
            types = np.concatenate([types, np.full(len(nk), wl.REQ_INSERT, np.uint8)])
            k = np.concatenate([k, nk])
            ln = np.concatenate([ln, nl])
            v = np.concatenate([v, rng.integers(0, 1 << 32, (len(nk), 2), dtype=np.uint64).astype(np.uint32)])
            vl = np.concatenate([vl, np.full(len(nk), 2, np.uint32)])
            gv, gl, gr = g.mixed(types, k, ln, v, vl)
            ov, ol, orr = o.mixed(types, k, ln, v, vl)
            nf = types != wl.REQ_FIND
            np.testing.assert_array_equal(gr[nf], orr[nf])
            assert_found(gv[~nf], gl[~nf], ov[~nf], ol[~nf], "mixed finds")
        ok, _, report = g.t.validate()
        assert ok, report
        same_state(g, o, 8, 2)
    finally:
        g.close()


@pytest.mark.parametrize("n", [1024, 3000, 100000])
def test_c2_batch_builds_links(n):
    """Keys that share their first slices (64 prefixes of 4 slices): layer 0 is
    built as 64 LINK entries and every key is inserted below them."""
    c2 = wl.C2(n_preload=n, n_prefixes=64)
    keys, lens, vals, vlens = c2.keys(np.arange(n))
    g, o = GpuIndex(tile_size=8, pool_bytes=1 << 30), OracleIndex()
    try:
        np.testing.assert_array_equal(g.insert(keys, lens, vals, vlens), o.insert(keys, lens, vals, vlens))
        ok, nkeys, report = g.t.validate()
        assert ok, report
        assert nkeys == n
        same_state(g, o, c2.maxK, c2.maxV)
    finally:
        g.close()


@pytest.mark.parametrize("n_first", [700, 5000])
def test_bulk_build_keeps_slice_pairs_together(n_first):
    """First slices that hold both a key ending there and keys continuing past
    it (two entries of one slice), mixed with slices holding one of the two,
    so that node bounds fall between such pairs; small batches below the old
    bulk threshold too.  Every key must be reachable."""
    rng = np.random.default_rng(n_first)
    firsts = np.unique(rng.integers(0, 1 << 32, 2 * n_first, dtype=np.uint64).astype(np.uint32))[:n_first]
    kind = rng.integers(0, 4, n_first)  # 0: ends only, 1: one continuing, 2: both, 3: ends + two continuing
    rows = []
    for s, k in zip(firsts, kind):
        if k in (0, 2, 3):
            rows.append((s, 0, 1))
        if k in (1, 2):
            rows.append((s, int(rng.integers(0, 1 << 32)), 2))
        if k == 3:
            rows.append((s, 5, 2))
            rows.append((s, 6, 2))
    rows = np.array(rows, dtype=np.uint64)
    rng.shuffle(rows)
    keys = rows[:, :2].astype(np.uint32)
    lens = rows[:, 2].astype(np.uint32)
    n = len(keys)
    vlens = rng.integers(1, 4, n).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, (n, 3), dtype=np.uint64).astype(np.uint32)
    vals[np.arange(3)[None, :] >= vlens[:, None]] = 0
    g, o = GpuIndex(tile_size=8, pool_bytes=256 << 20), OracleIndex()
    try:
        np.testing.assert_array_equal(g.insert(keys, lens, vals, vlens), o.insert(keys, lens, vals, vlens))
        ok, nkeys, report = g.t.validate()
        assert ok, report
        assert nkeys == n
        gv, gl = g.find(keys, lens, 3)
        ov, ol = o.find(keys, lens, 3)
        assert_found(gv, gl, ov, ol, "finds after a bulk build with slice pairs")
        same_state(g, o, 2, 3)
    finally:
        g.close()
