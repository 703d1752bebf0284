"""Parity with the oracle at the benchmark's own sizes.

The smaller parity tests (test_gpu_parity.py) run the same comparisons on trees
of at most 50K keys.  Here the trees have the benchmark's sizes and launch
shapes, where contention and tree depth are the benchmark's own:

* plain small workload: 1M keys of 1-8 slices with 2-slice values inserted
  into an empty tree (the bulk build), then 1M finds (half of them misses);
  every result, value length and value slice, then the full ordered contents;
* mixed workload: 16,777,216 preloaded keys of 2-16 slices under 4096 shared
  4-slice prefixes; four mixed batches of 1M requests reduced to their first
  request per key (so every request's result is defined), compared request by
  request; then four whole Zipf(0.99) batches of 1,048,576 requests, after
  which the full ordered contents and the structural check must match;
* range scan: 32M keys of 2 slices, then 1M scans of up to 100 results from
  random lower bounds: counts, keys, key lengths, values and value lengths.

Launch shapes are the benchmark's: finds at 8 lanes, writes at 32, scans at 4.
Integer results are compared exactly.  The oracle is the range-partitioned CPU
restatement, one thread per shard.
"""
import os
import time

import numpy as np
import pytest

from indexes import GpuIndex, OracleIndex
from indexingpu_b200 import workload as wl

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

THREADS = max(1, min(16, os.cpu_count() or 1))
STRIDE = 4096  # keys per scan query when whole contents are compared


def _index(pool_gb):
    g = GpuIndex(tile_size=8, pool_bytes=int(pool_gb * (1 << 30)))
    g.t.set_write_tile_size(32)
    g.t.set_scan_tile_size(4)
    return g


def _assert_rows(got_vals, got_vlens, exp_vals, exp_vlens, what):
    np.testing.assert_array_equal(got_vlens, exp_vlens, err_msg=f"{what}: value lengths")
    maxV = exp_vals.shape[1]
    live = np.arange(maxV)[None, :] < np.minimum(exp_vlens, maxV)[:, None]
    bad = np.nonzero(((got_vals != exp_vals) & live).any(axis=1))[0]
    assert len(bad) == 0, f"{what}: {len(bad)} rows with other value slices, first {bad[:5]}"


def assert_same_contents(g, o, maxK, maxV, what):
    """The tree holds exactly the oracle's keys and values: scans of STRIDE keys
    from every STRIDE-th oracle key must return the oracle's rows, a scan from
    the smallest key must start at the oracle's first key, and nothing may
    follow the oracle's last key."""
    ok_, okl, ov, ovl = o.dump(maxK, maxV)
    n = len(okl)
    assert n > 0
    starts = np.arange(0, n, STRIDE)
    counts, vals, vlens, keys, klens = g.scan(ok_[starts], okl[starts], STRIDE, maxV=maxV)
    exp_counts = np.minimum(STRIDE, n - starts).astype(np.uint32)
    np.testing.assert_array_equal(counts, exp_counts, err_msg=f"{what}: rows per chunk")
    take = (np.arange(STRIDE)[None, :] < exp_counts[:, None]).reshape(-1)
    np.testing.assert_array_equal(klens.reshape(-1)[take], okl, err_msg=f"{what}: key lengths")
    np.testing.assert_array_equal(keys.reshape(-1, maxK)[take], ok_, err_msg=f"{what}: keys")
    _assert_rows(vals.reshape(-1, maxV)[take], vlens.reshape(-1)[take], ov, ovl, what)
    # Nothing below the oracle's first key, nothing after its last.
    c0, _, _, k0, l0 = g.scan(np.zeros((1, maxK), np.uint32), np.ones(1, np.uint32), 1)
    assert c0[0] == 1 and l0[0, 0] == okl[0] and (k0[0, 0] == ok_[0]).all(), f"{what}: first key"
    c1, _, _, _, _ = g.scan(ok_[-1:], okl[-1:], 2)
    assert c1[0] == 1, f"{what}: keys after the oracle's last key"


def test_plain_1m_keys_then_1m_finds():
    t0 = time.time()
    w = wl.c1(n_keys=1 << 20, n_finds=1 << 20)
    g, o = _index(4), OracleIndex(shards=THREADS, threads=THREADS)
    try:
        rg = g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        ro = o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        np.testing.assert_array_equal(rg, ro)
        assert rg.all()
        vo, lo = o.find(w["find_keys"], w["find_lens"], 2)
        assert int((lo > 0).sum()) == int(w["find_hit"].sum())
        for conc in (False, True):
            vg, lg = g.find(w["find_keys"], w["find_lens"], 2, concurrent=conc)
            _assert_rows(vg, lg, vo, lo, f"1M finds (concurrent={conc})")
        assert_same_contents(g, o, 8, 2, "1M-key tree")
    finally:
        g.close()
    print(f"plain 1M: {time.time() - t0:.1f} s")


def test_mixed_16m_keys_touch_once_and_zipf_batches():
    t0 = time.time()
    c2 = wl.C2()  # 16,777,216 preloaded keys, 4096 prefixes, Zipf(0.99)
    keys, lens, vals, vlens = wl.keys_threaded(c2, np.arange(c2.n_preload), THREADS)
    g, o = _index(24), OracleIndex(shards=THREADS, threads=THREADS)
    try:
        rg = g.insert(keys, lens, vals, vlens)
        ro = o.insert(keys, lens, vals, vlens)
        np.testing.assert_array_equal(rg, ro)
        assert rg.all()
        del keys, lens, vals, vlens
        n = 1 << 20
        # Batches that touch each key once: every request's result is defined.
        for b in range(4):
            bt = c2.batch(b, n)
            _, first = np.unique(bt["ids"], return_index=True)
            bt = {k: v[np.sort(first)] for k, v in bt.items()}
            gv, gl, gr = g.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
            ov, ol, orr = o.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
            find = bt["types"] == wl.REQ_FIND
            np.testing.assert_array_equal(gr[~find], orr[~find], err_msg=f"batch {b}: write results")
            _assert_rows(gv[find], gl[find], ov[find], ol[find], f"batch {b}: finds")
            assert int((gl[find] > 0).sum()) > 0
        # Whole Zipf batches (repeated keys): the final contents are defined.
        for b in range(4, 8):
            bt = c2.batch(b, n)
            g.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
            o.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
        assert_same_contents(g, o, c2.maxK, c2.maxV, "16M-key tree after 8 batches")
        ok, nkeys, msg = g.t.validate()
        assert ok, msg
        assert nkeys == o.o.size()
    finally:
        g.close()
    print(f"mixed 16M: {time.time() - t0:.1f} s")


def test_scan_32m_keys_1m_queries():
    t0 = time.time()
    w = wl.c3(n_keys=1 << 25, n_queries=1 << 20)
    g, o = _index(12), OracleIndex(shards=THREADS, threads=THREADS)
    try:
        rg = g.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        ro = o.insert(w["keys"], w["lens"], w["vals"], w["vlens"])
        np.testing.assert_array_equal(rg, ro)
        assert rg.all()
        chunk = 1 << 17
        for q0 in range(0, len(w["lower"]), chunk):
            lo_k, lo_l = w["lower"][q0:q0 + chunk], w["lower_lens"][q0:q0 + chunk]
            cg, vg, vlg, kg, klg = g.scan(lo_k, lo_l, 100, maxV=1)
            co, vo, vlo, ko, klo = o.scan(lo_k, lo_l, 100, maxV=1)
            what = f"scans {q0}..{q0 + len(lo_l)}"
            np.testing.assert_array_equal(cg, co, err_msg=f"{what}: counts")
            np.testing.assert_array_equal(klg, klo, err_msg=f"{what}: key lengths")
            np.testing.assert_array_equal(kg, ko, err_msg=f"{what}: keys")
            np.testing.assert_array_equal(vlg, vlo, err_msg=f"{what}: value lengths")
            np.testing.assert_array_equal(vg, vo, err_msg=f"{what}: values")
            assert (cg == 100).mean() > 0.99
    finally:
        g.close()
    print(f"scan 32M: {time.time() - t0:.1f} s")
