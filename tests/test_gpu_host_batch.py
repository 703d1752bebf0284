"""mt_mixed_batch_host (host buffers, chunked, copies overlapped with the work)
against mt_mixed_batch with device buffers on an identical tree: per-request
results, find outputs and the final contents must match exactly.  Batches touch
every key once, so each request's result does not depend on the order in which
chunks are served."""
import numpy as np
import pytest

from indexingpu_b200 import workload as wl

pytestmark = pytest.mark.gpu
MAXK, MAXV = 16, 8
N_PRE = 20000


def _touch_once(bt):
    _, first = np.unique(bt["ids"], return_index=True)
    keep = np.sort(first)
    return {k: v[keep] for k, v in bt.items()}


def _trees(torch, c2, tile=8, write_tile=32):
    from indexingpu_b200 import GpuMasstree
    keys, lens, vals, vlens = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c2.keys(np.arange(N_PRE)))
    out = []
    for _ in range(2):
        t = GpuMasstree(pool_bytes=512 << 20, tile_size=tile)
        t.set_write_tile_size(write_tile)
        t.insert(keys, MAXK, lens, vals, MAXV, vlens, N_PRE)
        t.sync()
        out.append(t)
    return out


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


def _device_call(torch, tree, bt):
    d = {k: torch.from_numpy(np.ascontiguousarray(bt[k])).cuda() for k in ("types", "keys", "lens", "vals", "vlens")}
    res = torch.zeros(len(bt["types"]), dtype=torch.bool, device="cuda")
    tree.mixed_batch(d["types"], d["keys"], MAXK, d["lens"], d["vals"], MAXV, d["vlens"], res, len(bt["types"]))
    tree.sync()
    return d["vals"].cpu().numpy(), d["vlens"].cpu().numpy(), res.cpu().numpy()


def _host_buffers(torch, bt, with_lens=True, with_results=True):
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h = dict(types=pin(bt["types"]), keys=pin(bt["keys"]), lens=pin(bt["lens"]) if with_lens else None,
             vals=pin(bt["vals"]), vlens=pin(bt["vlens"]))
    h["res"] = torch.zeros(len(bt["types"]), dtype=torch.bool).pin_memory() if with_results else None
    return h


def _check(bt, got, exp, with_results=True):
    gv, gvl, gres = got
    ev, evl, eres = exp
    find = bt["types"] == wl.REQ_FIND
    if with_results:
        np.testing.assert_array_equal(gres[~find], eres[~find])
    np.testing.assert_array_equal(gvl[find], evl[find])
    for i in np.nonzero(find & (evl > 0))[0]:
        c = min(int(evl[i]), MAXV)
        assert np.array_equal(gv[i, :c], ev[i, :c]), i


@pytest.mark.parametrize("chunk", [1000, 0])
def test_host_batches_match_device_calls(chunk):
    """Two calls issued back to back (the second's uploads overlap the first's
    work), then one sync; chunks of 1000 wrap the three staging slots."""
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    ref, new = _trees(torch, c2)
    try:
        bts = [_touch_once(c2.batch(b, 5000)) for b in range(2)]
        exp = [_device_call(torch, ref, bt) for bt in bts]
        hs = [_host_buffers(torch, bt) for bt in bts]
        for bt, h in zip(bts, hs):
            new.mixed_batch_host(h["types"], h["keys"], MAXK, h["lens"], h["vals"], MAXV, h["vlens"], h["res"],
                                 len(bt["types"]), chunk=chunk)
        new.sync()
        for bt, h, e in zip(bts, hs, exp):
            _check(bt, (h["vals"].numpy(), h["vlens"].numpy(), h["res"].numpy()), e)
        n_final = N_PRE + 20000
        for x, y in zip(_dump(torch, ref, n_final), _dump(torch, new, n_final)):
            np.testing.assert_array_equal(x, y)
        ok, _, report = new.validate()
        assert ok, report
    finally:
        ref.close()
        new.close()


def test_host_batch_without_lengths_or_results():
    """NULL key lengths (every key has the maximum length) and NULL results."""
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    ref, new = _trees(torch, c2)
    try:
        bt = _touch_once(c2.batch(7, 3000))
        bt = dict(bt, lens=np.full(len(bt["types"]), MAXK, np.uint32))  # full-length rows (zero-padded keys)
        exp = _device_call(torch, ref, bt)
        h = _host_buffers(torch, bt, with_lens=False, with_results=False)
        new.mixed_batch_host(h["types"], h["keys"], MAXK, None, h["vals"], MAXV, h["vlens"], None, len(bt["types"]),
                             chunk=700)
        new.sync()
        _check(bt, (h["vals"].numpy(), h["vlens"].numpy(), None), exp, with_results=False)
        for x, y in zip(_dump(torch, ref, N_PRE + 3000), _dump(torch, new, N_PRE + 3000)):
            np.testing.assert_array_equal(x, y)
    finally:
        ref.close()
        new.close()


def test_host_batch_inputs_written_by_the_stream():
    """MT_FLAG_INPUTS_ON_STREAM: the host inputs are filled by copies queued on
    the same stream just before the call (from device tensors); the uploads
    must wait for them."""
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    ref, new = _trees(torch, c2)
    try:
        bt = _touch_once(c2.batch(11, 6000))
        exp = _device_call(torch, ref, bt)
        n = len(bt["types"])
        src = {k: torch.from_numpy(np.ascontiguousarray(bt[k])).cuda() for k in ("types", "keys", "lens", "vals",
                                                                              "vlens")}
        h = {k: torch.zeros_like(src[k], device="cpu").pin_memory() for k in src}
        res = torch.zeros(n, dtype=torch.bool).pin_memory()
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            torch.cuda._sleep(2_000_000)  # the copies below land well after the call is made
            for k in src:
                h[k].copy_(src[k], non_blocking=True)
        new.mixed_batch_host(h["types"], h["keys"], MAXK, h["lens"], h["vals"], MAXV, h["vlens"], res, n, stream=s,
                             inputs_on_stream=True)
        new.sync(s)
        _check(bt, (h["vals"].numpy(), h["vlens"].numpy(), res.numpy()), exp)
    finally:
        ref.close()
        new.close()
