"""The eleven scenarios of IndexinGPU's masstree unit test
(test/unittest_masstree.cu:318-708), restated over the numpy adapters in
indexes.py.  Expected results are the reference test's own closed-form
expectations computed from the seeded inputs in tests/golden/.

Each scenario takes a factory returning a fresh index and the golden input
dict; it raises AssertionError on a mismatch.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHAPES = ["k1-1_v1-1", "k1-200_v1-1", "k1-1_v1-200", "k1-200_v1-200"]
REQ_INSERT, REQ_ERASE, REQ_FIND, REQ_UPDATE = 0, 1, 2, 3


def load_inputs(shape, duplicate=False):
    d = dict(np.load(os.path.join(GOLDEN, f"unittest_inputs_{shape}.npz")))
    if duplicate:
        # testing_input(..., duplicate=true): the second half repeats the first
        # (test/unittest_masstree.cu:125-140).
        n = len(d["lengths"])
        h = (n + 1) // 2
        for name in ("keys", "keys_not_exist", "values", "values2", "lengths", "value_lengths"):
            a = d[name].copy()
            a[h:] = a[: n - h]
            d[name] = a
    return d


def assert_found(vals, vlens, exp_vals, exp_vlens, what):
    np.testing.assert_array_equal(vlens, exp_vlens, err_msg=f"{what}: value lengths")
    maxV = vals.shape[1]
    for i in np.nonzero(exp_vlens)[0]:
        c = min(int(exp_vlens[i]), maxV)
        if not np.array_equal(vals[i, :c], exp_vals[i, :c]):
            raise AssertionError(f"{what}: value of item {i}: {vals[i, :c]} != {exp_vals[i, :c]}")


def _ins(idx, d, n=None):
    return idx.insert(d["keys"], d["lengths"], d["values"], d["value_lengths"], n)


def validate(make, d):
    """Validate: insert all, then the index in key order equals the sorted input."""
    idx = make()
    _ins(idx, d)
    n = len(d["lengths"])
    order = sorted(range(n), key=lambda i: tuple(d["keys"][i, : d["lengths"][i]]))
    first = d["keys"][order[0]][None, :]
    counts, vals, vlens, okeys, oklens = idx.scan(first, d["lengths"][order[:1]], n + 4, maxV=d["values"].shape[1])
    assert counts[0] == n, f"full scan saw {counts[0]} of {n} keys"
    for r, i in enumerate(order):
        L = d["lengths"][i]
        assert oklens[0, r] == L and np.array_equal(okeys[0, r, :L], d["keys"][i, :L]), f"order breaks at rank {r}"
        assert vlens[0, r] == d["value_lengths"][i]


def find_exist(make, d):
    idx = make()
    _ins(idx, d)
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert_found(vals, vlens, d["values"], d["value_lengths"], "FindExist")


def find_not_exist(make, d):
    idx = make()
    _ins(idx, d)
    vals, vlens = idx.find(d["keys_not_exist"], d["lengths"], d["values"].shape[1])
    assert not vlens.any(), "FindNotExist: a missing key was found"


def update(make, d):
    idx = make()
    _ins(idx, d)
    res = idx.update(d["keys"], d["lengths"], d["values2"], d["value_lengths"])
    if res is not None:
        assert res.all(), "Update: an existing key was not updated"
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert_found(vals, vlens, d["values2"], d["value_lengths"], "Update")


def erase_all(make, d):
    idx = make()
    _ins(idx, d)
    res = idx.erase(d["keys"], d["lengths"])
    if res is not None:
        assert res.all(), "EraseAll: an erase of a present key failed"
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert not vlens.any(), "EraseAll: an erased key was found"


def erase_none(make, d):
    idx = make()
    _ins(idx, d)
    res = idx.erase(d["keys_not_exist"], d["lengths"])
    if res is not None:
        assert not res.any(), "EraseNone: an erase of a missing key succeeded"
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert_found(vals, vlens, d["values"], d["value_lengths"], "EraseNone")


def insert_twice_erase_all(make, d):
    """Input with duplicated second half: insert all, erase all, find nothing."""
    idx = make()
    res = _ins(idx, d)
    n = len(d["lengths"])
    h = (n + 1) // 2
    if res is not None:
        dup = n - h
        # Each duplicated key is inserted twice in one batch: exactly one wins.
        assert (res[:dup].astype(int) + res[h:h + dup].astype(int) == 1).all()
        assert res[dup:h].all()
    idx.erase(d["keys"], d["lengths"])
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert not vlens.any(), "InsertTwiceEraseAll: a key survived"


def erase_all_insert_all(make, d):
    idx = make()
    _ins(idx, d)
    idx.erase(d["keys"], d["lengths"])
    res = _ins(idx, d)
    if res is not None:
        assert res.all(), "EraseAllInsertAll: a re-insert failed"
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1])
    assert_found(vals, vlens, d["values"], d["value_lengths"], "EraseAllInsertAll")


def erase_all_twice(make, d):
    """Duplicated input: insert the first half, erase all n (duplicates twice)."""
    idx = make()
    n = len(d["lengths"])
    h = n // 2
    _ins(idx, d, h)
    res = idx.erase(d["keys"], d["lengths"])
    if res is not None:
        hh = (n + 1) // 2
        dup = n - hh
        # Every first-half key is erased exactly once across its two requests.
        assert (res[:dup].astype(int) + res[hh:].astype(int) == 1).all()
    vals, vlens = idx.find(d["keys"], d["lengths"], d["values"].shape[1], n=h)
    assert not vlens[:h].any(), "EraseAllTwice: a key survived"


def range_query(make, d, max_count=10):
    """RangeQuery: queries [key[b], key[e]] over the sorted input
    (test/unittest_masstree.cu:230-304, 522-569)."""
    n = len(d["lengths"])
    order = sorted(range(n), key=lambda i: tuple(d["keys"][i, : d["lengths"][i]]))
    keys, lens = d["keys"][order], d["lengths"][order]
    vals, vlens = d["values"][order], d["value_lengths"][order]
    nq = n // 2
    b = np.arange(nq) % n
    cnt = 1 + (np.arange(nq) % (2 * max_count))
    e = np.minimum(b + cnt - 1, n - 1)
    exp_counts = np.minimum(e - b + 1, max_count)
    idx = make()
    idx.insert(keys, lens, vals, vlens)
    counts, ovals, ovlens, okeys, oklens = idx.scan(keys[b], lens[b], max_count, keys[e], lens[e],
                                                    maxV=vals.shape[1])
    np.testing.assert_array_equal(counts, exp_counts, err_msg="RangeQuery counts")
    maxV = vals.shape[1]
    for q in range(nq):
        for v in range(exp_counts[q]):
            src = b[q] + v
            assert ovlens[q, v] == vlens[src], f"RangeQuery q{q} r{v} value length"
            c = min(int(vlens[src]), maxV)
            assert np.array_equal(ovals[q, v, :c], vals[src, :c]), f"RangeQuery q{q} r{v} value"
            assert oklens[q, v] == lens[src], f"RangeQuery q{q} r{v} key length"
            assert np.array_equal(okeys[q, v, : lens[src]], keys[src, : lens[src]]), f"RangeQuery q{q} r{v} key"


def concurrent_mix(make, d):
    """ConcurrentMix: A/B/C/D quarters of the shuffled input in one shuffled
    mixed batch (test/unittest_masstree.cu:571-708)."""
    n = len(d["lengths"])
    o = d["shuffle_order"]
    keys, lens = d["keys"][o], d["lengths"][o]
    vals, vals2, vlens = d["values"][o], d["values2"][o], d["value_lengths"][o]
    q = n // 4
    A, B, C, D = 0, q, 2 * q, 3 * q
    m = 10 * q
    perm = d["mix_order"]
    maxK, maxV = keys.shape[1], vals.shape[1]
    types = np.zeros(m, np.uint8)
    mk = np.zeros((m, maxK), np.uint32)
    ml = np.zeros(m, np.uint32)
    mv = np.zeros((m, maxV), np.uint32)
    mvl = np.zeros(m, np.uint32)
    inv = np.zeros(m, np.int64)
    plan = [(A, REQ_INSERT), (C, REQ_INSERT), (A, REQ_UPDATE), (D, REQ_UPDATE), (A, REQ_FIND), (B, REQ_FIND),
            (C, REQ_FIND), (D, REQ_FIND), (B, REQ_ERASE), (D, REQ_ERASE)]
    for blk, (src0, kind) in enumerate(plan):
        for i in range(q):
            dst = perm[blk * q + i]
            src = src0 + i
            types[dst] = kind
            mk[dst] = keys[src]
            ml[dst] = lens[src]
            if kind in (REQ_INSERT, REQ_UPDATE):
                mv[dst] = vals[src] if kind == REQ_INSERT else vals2[src]
                mvl[dst] = vlens[src]
            inv[dst] = blk * q + i
    idx = make()
    idx.insert(keys, lens, vals, vlens, n=2 * q)
    ov, ovl, res = idx.mixed(types, mk, ml, mv, mvl)
    for i in range(m):
        dst = inv[i]
        blk, off = divmod(int(dst), q)
        if blk in (0, 1):
            assert res[i] == (1 if blk == 1 else 0), f"ConcurrentMix insert {dst}"
        elif blk in (2, 3):
            assert res[i] == (1 if blk == 2 else 0), f"ConcurrentMix update {dst}"
        elif blk == 4:
            assert ovl[i] == vlens[A + off], f"ConcurrentMix find A {dst}"
            c = min(int(vlens[A + off]), maxV)
            got = ov[i, :c]
            assert np.array_equal(got, vals[A + off, :c]) or np.array_equal(got, vals2[A + off, :c])
        elif blk == 7:
            assert ovl[i] == 0, f"ConcurrentMix find D {dst}"
        elif blk == 8:
            assert res[i] == 1, f"ConcurrentMix erase B {dst}"
        elif blk == 9:
            assert res[i] == 0, f"ConcurrentMix erase D {dst}"
    fv, fvl = idx.find(keys, lens, maxV, n=4 * q)
    exp_l = np.where((np.arange(4 * q) < q) | ((np.arange(4 * q) >= 2 * q) & (np.arange(4 * q) < 3 * q)),
                     vlens[: 4 * q], 0)
    exp_v = np.where((np.arange(4 * q) < q)[:, None], vals2[: 4 * q], vals[: 4 * q])
    assert_found(fv, fvl, exp_v, exp_l, "ConcurrentMix final find")


def _dup(fn):
    def run(make, d):
        return fn(make, d)
    run.duplicate = True
    return run


SCENARIOS = {
    "Validate": validate,
    "FindExist": find_exist,
    "FindNotExist": find_not_exist,
    "Update": update,
    "EraseAll": erase_all,
    "EraseNone": erase_none,
    "InsertTwiceEraseAll": _dup(insert_twice_erase_all),
    "EraseAllInsertAll": erase_all_insert_all,
    "EraseAllTwice": _dup(erase_all_twice),
    "RangeQuery": range_query,
    "ConcurrentMix": concurrent_mix,
}


def run_scenario(name, shape, make):
    fn = SCENARIOS[name]
    d = load_inputs(shape, duplicate=getattr(fn, "duplicate", False))
    fn(make, d)
