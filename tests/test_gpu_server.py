"""Online serving (mt_server_start / submit / poll / stop).

Requests live in host memory; a client thread submits them one by one while
earlier ones are still on the device, and the main thread polls their tickets.
Every op of the stream touches its own key (workload.serve_stream with
disjoint=True), so each op's result is defined independently of how requests
interleave: the oracle applied to the whole stream gives the expected result of
every op, which is also what each request gets served alone.  The stream is
served (a) request by request, each alone (submit, wait, next), and (b) with a
client thread submitting while the loop runs and the staging ring small enough
to wrap and to make admission wait; both must equal the oracle op by op and
leave the oracle's contents.
"""
import threading
import time

import numpy as np
import pytest

from indexes import OracleIndex, same_state
from indexingpu_b200 import workload as wl

pytestmark = pytest.mark.gpu
MAXK, MAXV = 16, 8
N_PRE = 40000


def _setup(torch, c2, tile=8):
    from indexes import GpuIndex
    g = GpuIndex(tile_size=tile, pool_bytes=256 << 20)
    g.t.set_write_tile_size(32)
    k, l, v, vl = c2.keys(np.arange(N_PRE))
    g.insert(k, l, v, vl)
    o = OracleIndex()
    o.insert(k, l, v, vl)
    return g, o


def _host(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory()


def _serve_online(torch, g, st, alone, **cfg):
    from indexingpu_b200.masstree import MasstreeServer
    types, keys, lens = _host(torch, st["types"]), _host(torch, st["keys"]), _host(torch, st["lens"])
    vals, vlens = _host(torch, st["vals"]), _host(torch, st["vlens"])
    res = torch.zeros(len(st["types"]), dtype=torch.bool).pin_memory()
    first, nops = st["first"], st["nops"]
    n_req = len(nops)
    srv = MasstreeServer(g.t, MAXK, MAXV, **cfg)
    tickets = [None] * n_req
    lat = np.zeros(n_req, np.uint64)
    try:
        def submit(r):
            f, n = int(first[r]), int(nops[r])
            return srv.submit(types[f:f + n], keys[f:f + n], lens[f:f + n], vals[f:f + n], vlens[f:f + n],
                              res[f:f + n], n)

        def wait(r, limit=60.0):
            t0 = time.time()
            while True:
                done, ns = srv.poll(tickets[r])
                if done:
                    lat[r] = ns
                    return
                assert time.time() - t0 < limit, f"request {r} not done"

        if alone:
            for r in range(n_req):
                tickets[r] = submit(r)
                wait(r)
        else:
            def client():
                for r in range(n_req):
                    tickets[r] = submit(r)
                    if r % 16 == 15:
                        time.sleep(0.0005)  # later requests arrive while earlier ones run

            th = threading.Thread(target=client)
            th.start()
            for r in range(n_req):
                while tickets[r] is None:
                    time.sleep(0)
                wait(r)
            th.join()
        # Stage sums: every request counted once, each stage's sum within the
        # sum of the requests' latencies.
        sst = srv.stats()
        assert sst["requests"] == n_req and sst["ops"] == int(nops.sum()), sst
        stages = sst["queued_ns"] + sst["upload_ns"] + sst["device_ns"] + sst["deliver_ns"]
        assert 0 < stages <= int(lat.sum()) + n_req * 1000, (sst, int(lat.sum()))
        assert sst["max_latency_ns"] >= int(lat.max()), (sst, int(lat.max()))
    finally:
        srv.stop()
    return vals.numpy(), vlens.numpy(), res.numpy().astype(np.uint8), lat


def _check(st, got, exp):
    gv, gvl, gres, _ = got
    ev, evl, eres = exp
    find = st["types"] == wl.REQ_FIND
    np.testing.assert_array_equal(gres[~find], eres[~find])
    np.testing.assert_array_equal(gvl[find], evl[find])
    live = np.arange(MAXV)[None, :] < np.minimum(evl, MAXV)[:, None]
    bad = np.nonzero(((gv != ev) & live & find[:, None]).any(axis=1))[0]
    assert len(bad) == 0, bad[:5]


@pytest.mark.parametrize("tile,chunk", [(8, 0), (16, 4)])
def test_online_server_alone_and_in_the_mix(tile, chunk):
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    st = wl.serve_stream(c2, 300, rate_per_s=None, min_ops=1, max_ops=200, disjoint=True, seed=0xC5 + tile)
    _, o0 = _setup(torch, c2, tile)
    exp = o0.mixed(st["types"], st["keys"], st["lens"], st["vals"], st["vlens"])
    for alone in (True, False):
        g, o = _setup(torch, c2, tile)
        try:
            # In the mix: a staging ring of 2048 ops and 32 request slots, so
            # the ring wraps and admission waits for earlier requests.
            cfg = dict(chunk_ops=chunk) if alone else dict(chunk_ops=chunk, max_ops_in_flight=2048,
                                                           max_requests_in_flight=32)
            t0 = time.time()
            got = _serve_online(torch, g, st, alone, **cfg)
            print(f"tile {tile} chunk {chunk} alone={alone}: {time.time() - t0:.3f} s, "
                  f"latency p50 {np.percentile(got[3], 50) / 1e3:.1f} us, max {got[3].max() / 1e3:.1f} us")
            _check(st, got, exp)
            assert (got[3] > 0).all()
            o.mixed(st["types"], st["keys"], st["lens"], st["vals"], st["vlens"])
            same_state(g, o, MAXK, MAXV)
            ok, nkeys, msg = g.t.validate()
            assert ok and nkeys == o.o.size(), msg
        finally:
            g.close()


def test_online_server_rejects_bad_requests():
    import torch
    from indexingpu_b200 import MasstreeError
    from indexingpu_b200.masstree import MasstreeServer
    c2 = wl.C2(n_preload=1000, n_prefixes=8)
    from indexes import GpuIndex
    g = GpuIndex(tile_size=8, pool_bytes=64 << 20)
    try:
        srv = MasstreeServer(g.t, MAXK, MAXV, max_ops_in_flight=64)
        try:
            buf = torch.zeros(128 * MAXK, dtype=torch.uint32).pin_memory()
            with pytest.raises(MasstreeError):
                srv.submit(buf, buf, None, buf, buf, None, 0)  # no ops
            with pytest.raises(MasstreeError):
                srv.submit(buf, buf, None, buf, buf, None, 65)  # more than the staging holds
            with pytest.raises(MasstreeError):
                srv.poll(5)  # no such ticket
        finally:
            srv.stop()
    finally:
        g.close()
    del c2


def test_online_replay_of_a_timed_stream():
    # mt_serve in MT_SERVE_ONLINE mode: host buffers, submitted at Poisson
    # arrival times through the server API; results as the oracle's.
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    st = wl.serve_stream(c2, 400, rate_per_s=2e4, min_ops=1, max_ops=128, disjoint=True, seed=0xC55)
    g, o = _setup(torch, c2, 8)
    try:
        exp = o.mixed(st["types"], st["keys"], st["lens"], st["vals"], st["vlens"])
        h = {k: _host(torch, st[k]) for k in ("types", "keys", "lens", "vals", "vlens")}
        res = torch.zeros(len(st["types"]), dtype=torch.bool).pin_memory()
        lat, stats = g.t.serve(h["types"], h["keys"], MAXK, h["lens"], h["vals"], MAXV, h["vlens"], res,
                               st["first"], st["nops"], st["arrival_ns"], online=True)
        assert stats["requests_done"] == 400 and (lat > 0).all()
        assert 0 < sum(stats["stage_ns"].values()) <= int(lat.sum()) + 400 * 1000, stats
        _check(st, (h["vals"].numpy(), h["vlens"].numpy(), res.numpy().astype(np.uint8), lat), exp)
        same_state(g, o, MAXK, MAXV)
    finally:
        g.close()
