"""Failure detection without a GPU fault.

* Bounded lock waits: a node lock that is never released (set from the host
  with mt_inject_node_lock, as a writer that died holding it would leave it)
  makes the next writer give up after mt_set_lock_wait attempts and the call
  report MT_ERR_LOCK_TIMEOUT; the context stays usable, the tree unchanged,
  and the same request succeeds once the lock is gone.  The reference spins on
  such a lock without a bound (include/masstree_node_subwarp.hpp:217-219).
* The 128-byte line self-test (mt_selftest_line_atomicity) that motivates the
  node checksums runs, bounded by its iteration count, at every tile width.
"""
import numpy as np
import pytest

from indexes import GpuIndex, OracleIndex
from indexingpu_b200 import MasstreeError
from indexingpu_b200.masstree import line_atomicity_selftest
from indexingpu_b200 import workload as wl

pytestmark = pytest.mark.gpu

MT_ERR_LOCK_TIMEOUT = 2


@pytest.mark.parametrize("tile", [8, 32])
def test_lock_timeout_reported_and_recovered(tile):
    # Ten keys with distinct first slices fit in the root border node (slab 0),
    # so every insert or update below has to lock that node.
    w = wl.c1(n_keys=20, n_finds=10)
    keys, lens, vals, vlens = w["keys"], w["lens"], w["vals"], w["vlens"]
    assert len(np.unique(keys[:, 0])) == 20
    g, o = GpuIndex(tile, pool_bytes=64 << 20), OracleIndex()
    try:
        assert g.insert(keys[:10], lens[:10], vals[:10], vlens[:10]).all()
        o.insert(keys[:10], lens[:10], vals[:10], vlens[:10])
        assert g.t.stats()["used_slabs"] <= 11  # the root and ten value chains: no split yet
        g.t.set_lock_wait(2000)
        g.t.inject_node_lock(0, True)
        with pytest.raises(MasstreeError) as ei:
            g.insert(keys[10:], lens[10:], vals[10:], vlens[10:])
        assert ei.value.code == MT_ERR_LOCK_TIMEOUT
        new_vals = vals[:10] ^ np.uint32(0x5A5A5A5A)
        with pytest.raises(MasstreeError) as ei:
            g.update(keys[:10], lens[:10], new_vals, vlens[:10])
        assert ei.value.code == MT_ERR_LOCK_TIMEOUT
        # Lock-free finds still work while the lock is held, and see nothing
        # of the calls that timed out.
        vg, lg = g.find(keys, lens, 2)
        vo, lo = o.find(keys, lens, 2)
        np.testing.assert_array_equal(lg, lo)
        np.testing.assert_array_equal(vg, vo)
        g.t.inject_node_lock(0, False)
        ok, nkeys, msg = g.t.validate()
        assert ok and nkeys == 10, msg
        # The same requests succeed once the lock is gone.
        np.testing.assert_array_equal(g.insert(keys[10:], lens[10:], vals[10:], vlens[10:]),
                                      o.insert(keys[10:], lens[10:], vals[10:], vlens[10:]))
        np.testing.assert_array_equal(g.update(keys[:10], lens[:10], new_vals, vlens[:10]),
                                      o.update(keys[:10], lens[:10], new_vals, vlens[:10]))
        ok, nkeys, msg = g.t.validate()
        assert ok and nkeys == 20, msg
        vg, lg = g.find(keys, lens, 2)
        vo, lo = o.find(keys, lens, 2)
        np.testing.assert_array_equal(lg, lo)
        np.testing.assert_array_equal(vg, vo)
    finally:
        g.close()


@pytest.mark.parametrize("tile", [4, 8, 16, 32])
def test_line_atomicity_selftest_runs_bounded(tile):
    iters = 2000
    reads, torn = line_atomicity_selftest(tile, nlines=64, iters=iters)
    # Half the tiles of 8 blocks of 128 threads per SM read, each `iters` times.
    assert reads > 0 and reads % iters == 0
    assert 0 <= torn <= reads
    print(f"line self-test tile {tile}: {reads} reads, {torn} torn")
