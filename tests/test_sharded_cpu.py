"""The range-sharded form (indexingpu_b200/sharded.py) on gloo ranks on CPU.

Each rank's shard is a small in-test ordered map (the exchange logic is what
is under test here; the GPU shard is covered by the GPU test of this file's
twin).  Every rank submits its own requests; the union of all ranks' results
must equal the oracle's on the union of the requests: inserts of a preload,
a mixed batch that touches every key once, and scans that cross shard
boundaries (the next shard continues from its smallest key).
"""
import bisect
import os
import socket

import numpy as np
import pytest

MAXK, MAXV = 16, 8


class DictShard:
    """An ordered map of u32-slice tuples (a key that is a prefix of another
    sorts first, as in the reference), with the local-shard interface."""

    def __init__(self):
        self.keys, self.vals = [], []

    def _find(self, k):
        i = bisect.bisect_left(self.keys, k)
        return i, i < len(self.keys) and self.keys[i] == k

    def mixed(self, types, keys, klens, vals, vlens):
        import torch
        t, k, kl, v, vl = (x.cpu().numpy() for x in (types, keys.view(torch.int32), klens.view(torch.int32),
                                                       vals.view(torch.int32), vlens.view(torch.int32)))
        k, kl, v, vl = k.view(np.uint32), kl.view(np.uint32), v.view(np.uint32).copy(), vl.view(np.uint32).copy()
        res = np.zeros(len(t), bool)
        for r in range(len(t)):
            key = tuple(int(x) for x in k[r, : kl[r]])
            i, hit = self._find(key)
            if t[r] == 0:  # insert
                if not hit:
                    self.keys.insert(i, key)
                    self.vals.insert(i, tuple(int(x) for x in v[r, : vl[r]]))
                res[r] = not hit
            elif t[r] == 1:  # erase
                if hit:
                    del self.keys[i], self.vals[i]
                res[r] = hit
            elif t[r] == 3:  # update
                if hit:
                    self.vals[i] = tuple(int(x) for x in v[r, : vl[r]])
                res[r] = hit
            else:  # find
                val = self.vals[i] if hit else ()
                vl[r] = len(val)
                for j, x in enumerate(val[:MAXV]):
                    v[r, j] = x
        tt = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).view(torch.uint32)  # noqa: E731
        return tt(v), tt(vl), torch.from_numpy(res)

    def scan(self, lower, lower_lens, max_count, maxV):
        import torch
        lo, ll = lower.view(torch.int32).numpy().view(np.uint32), lower_lens.view(torch.int32).numpy().view(np.uint32)
        nq, maxK = lo.shape
        counts = np.zeros(nq, np.uint32)
        vals = np.zeros((nq, max_count, maxV), np.uint32)
        vlens = np.zeros((nq, max_count), np.uint32)
        keys = np.zeros((nq, max_count, maxK), np.uint32)
        klens = np.zeros((nq, max_count), np.uint32)
        for q in range(nq):
            i = bisect.bisect_left(self.keys, tuple(int(x) for x in lo[q, : ll[q]]))
            c = 0
            while i < len(self.keys) and c < max_count:
                key, val = self.keys[i], self.vals[i]
                keys[q, c, : len(key)] = key
                klens[q, c] = len(key)
                vals[q, c, : min(len(val), maxV)] = val[:maxV]
                vlens[q, c] = len(val)
                c += 1
                i += 1
            counts[q] = c
        tt = lambda a: torch.from_numpy(a.view(np.int32)).view(torch.uint32)  # noqa: E731
        return tt(counts), tt(vals), tt(vlens), tt(keys), tt(klens)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _t(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    from indexingpu_b200 import workload as wl
    from indexingpu_b200.sharded import ShardedMasstree
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = ShardedMasstree(DictShard(), MAXK, MAXV)
        c2 = wl.C2(n_preload=3000, n_prefixes=64)
        # Preload: every rank inserts its own third of the keys.
        ids = np.arange(rank, 3000, world)
        k, l, v, vl = c2.keys(ids)
        _, _, res = sh.mixed_batch(_t(np.zeros(len(ids), np.uint8)), _t(k), _t(l), _t(v), _t(vl))
        assert res.all()
        # A mixed batch touching every key once, split over the ranks.
        bt = c2.batch(0, 2000)
        _, first = np.unique(bt["ids"], return_index=True)
        keep = np.sort(first)
        mine = keep[rank::world]
        gv, gl, gr = sh.mixed_batch(_t(bt["types"][mine]), _t(bt["keys"][mine]), _t(bt["lens"][mine]),
                                    _t(bt["vals"][mine]), _t(bt["vlens"][mine]))
        # Scans from every rank, from present and absent lower bounds, long
        # enough to cross shard boundaries.
        lo_ids = np.arange(rank, 3000, 97)
        lk, ll, _, _ = c2.keys(lo_ids)
        sc = sh.scan(_t(lk), _t(ll), 1200)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), mine=mine, gv=gv.view(torch.int32).numpy(),
                 gl=gl.view(torch.int32).numpy(), gr=gr.numpy(), lo_ids=lo_ids,
                 **{f"s{j}": x.view(torch.int32).numpy() for j, x in enumerate(sc)})
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_mixed_and_scan_match_oracle(world, tmp_path):
    import torch.multiprocessing as mp

    from indexes import OracleIndex
    from indexingpu_b200 import workload as wl
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    c2 = wl.C2(n_preload=3000, n_prefixes=64)
    o = OracleIndex()
    k, l, v, vl = c2.keys(np.arange(3000))
    o.insert(k, l, v, vl)
    bt = c2.batch(0, 2000)
    _, first = np.unique(bt["ids"], return_index=True)
    keep = np.sort(first)
    ev, evl, eres = o.mixed(bt["types"][keep], bt["keys"][keep], bt["lens"][keep], bt["vals"][keep],
                            bt["vlens"][keep])
    pos = {int(j): n for n, j in enumerate(keep)}
    seen = 0
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        for a, j in enumerate(d["mine"]):
            e = pos[int(j)]
            if bt["types"][j] == wl.REQ_FIND:
                assert d["gl"][a] == evl[e]
                c = min(int(evl[e]), MAXV)
                assert np.array_equal(d["gv"][a, :c].view(np.uint32), ev[e, :c])
            else:
                assert bool(d["gr"][a]) == bool(eres[e])
            seen += 1
        lk, ll, _, _ = c2.keys(d["lo_ids"])
        exp = o.scan(lk, ll, 1200, maxV=MAXV)
        got = [d[f"s{j}"].view(np.uint32) for j in range(5)]
        for x, y, name in zip(got, exp, ["counts", "values", "value lengths", "keys", "key lengths"]):
            np.testing.assert_array_equal(x, y, err_msg=f"rank {r} scan {name}")
    assert seen == len(keep)
