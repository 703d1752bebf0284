"""mt_mixed_batch_noalloc: the mixed batch for callers that cannot allocate
device memory during the call (request loops that must never wait for the
driver's allocator, programs that give the whole device to the slab pool or to
another allocator up front).  It must give exactly
the results of mt_mixed_batch: two identical trees, two mixed batches in a row,
one tree driven through each entry point, compared request by request and by
final contents.  Collected last so a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAXK, MAXV = 16, 8
NOALLOC_MAX = 1 << 18


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _touch_once(bt):
    _, first = np.unique(bt["ids"], return_index=True)
    keep = np.sort(first)
    return {k: v[keep] for k, v in bt.items()}


def _dump(tree, torch, n):
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
    return c, keys[0, :c].cpu().numpy(), klens[0, :c].cpu().numpy(), vals[0, :c].cpu().numpy(), \
        vlens[0, :c].cpu().numpy()


def test_noalloc_mixed_batch_matches_mixed_batch():
    import torch

    from indexingpu_b200 import GpuMasstree, _lib
    from indexingpu_b200 import workload as wl

    lib = _lib.load()
    c2 = wl.C2(n_preload=30000, n_prefixes=64)
    keys, lens, vals, vlens = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c2.keys(np.arange(30000)))
    ref = GpuMasstree(pool_bytes=256 << 20, tile_size=16)
    new = GpuMasstree(pool_bytes=256 << 20, tile_size=16)
    try:
        for t in (ref, new):
            t.set_write_tile_size(32)
            t.insert(keys, MAXK, lens, vals, MAXV, vlens, 30000)
            t.sync()
        for b in range(2):  # two calls in a row
            bt = _touch_once(c2.batch(b, 20000))
            n = len(bt["types"])
            d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in bt.items() if k != "ids"}
            rv, rl = d["vals"].clone(), d["vlens"].clone()
            rr = torch.zeros(n, dtype=torch.bool, device="cuda")
            ref.mixed_batch(d["types"], d["keys"], MAXK, d["lens"], rv, MAXV, rl, rr, n)
            ref.sync()
            nv, nl = d["vals"].clone(), d["vlens"].clone()
            nr = torch.zeros(n, dtype=torch.bool, device="cuda")
            rc = lib.mt_mixed_batch_noalloc(new._h, _ptr(d["types"]), _ptr(d["keys"]), MAXK, _ptr(d["lens"]),
                                            _ptr(nv), MAXV, _ptr(nl), _ptr(nr), n, None)
            assert rc == 0, rc
            new.sync()
            types = bt["types"]
            find = types == wl.REQ_FIND
            np.testing.assert_array_equal(nr.cpu().numpy()[~find], rr.cpu().numpy()[~find])
            gl, el = nl.cpu().numpy(), rl.cpu().numpy()
            np.testing.assert_array_equal(gl[find], el[find])
            gv, ev = nv.cpu().numpy(), rv.cpu().numpy()
            for i in np.nonzero(find & (el > 0))[0]:
                c = min(int(el[i]), MAXV)
                assert np.array_equal(gv[i, :c], ev[i, :c]), i
        a = _dump(ref, torch, 120000)
        b = _dump(new, torch, 120000)
        assert a[0] == b[0]
        for x, y in zip(a[1:], b[1:]):
            np.testing.assert_array_equal(x, y)
        # Beyond the fixed scratch: refused before anything is launched.
        big = NOALLOC_MAX + 1
        rc = lib.mt_mixed_batch_noalloc(new._h, _ptr(d["types"]), _ptr(d["keys"]), MAXK, _ptr(d["lens"]), _ptr(nv),
                                        MAXV, _ptr(nl), _ptr(nr), big, None)
        assert rc == 8  # MT_ERR_BATCH_TOO_LARGE
        new.sync()
    finally:
        ref.close()
        new.close()
