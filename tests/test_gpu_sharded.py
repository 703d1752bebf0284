"""The range-sharded form over GPU shards (GpuShard: the CUDA tree behind
mt_mixed_batch / mt_scan) with NCCL, on the one GPU a test box has (world
size 1: every exchange is the NCCL all-to-all of a single rank).  The
exchange logic across several ranks is covered on CPU by test_sharded_cpu.py.
"""
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MAXK, MAXV = 16, 8


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_gpu_shard_matches_oracle():
    import torch
    import torch.distributed as dist

    from indexes import GpuIndex, OracleIndex
    from indexingpu_b200 import workload as wl
    from indexingpu_b200.sharded import GpuShard, ShardedMasstree
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    g = GpuIndex(tile_size=8, pool_bytes=256 << 20)
    try:
        g.t.set_write_tile_size(32)
        sh = ShardedMasstree(GpuShard(g.t), MAXK, MAXV)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        c2 = wl.C2(n_preload=20000, n_prefixes=64)
        k, l, v, vl = c2.keys(np.arange(20000))
        o = OracleIndex()
        o.insert(k, l, v, vl)
        _, _, res = sh.mixed_batch(d(np.zeros(20000, np.uint8)), d(k), d(l), d(v), d(vl))
        assert bool(res.all())
        bt = c2.batch(0, 8000)
        _, first = np.unique(bt["ids"], return_index=True)
        bt = {key: x[np.sort(first)] for key, x in bt.items()}
        gv, gl, gr = sh.mixed_batch(d(bt["types"]), d(bt["keys"]), d(bt["lens"]), d(bt["vals"]), d(bt["vlens"]))
        ev, evl, eres = o.mixed(bt["types"], bt["keys"], bt["lens"], bt["vals"], bt["vlens"])
        find = bt["types"] == wl.REQ_FIND
        gv, gl, gr = gv.cpu().numpy(), gl.cpu().numpy(), gr.cpu().numpy()
        np.testing.assert_array_equal(gr[~find].astype(np.uint8), eres[~find])
        np.testing.assert_array_equal(gl[find], evl[find])
        live = np.arange(MAXV)[None, :] < np.minimum(evl, MAXV)[:, None]
        assert not ((gv != ev) & live & find[:, None]).any()
        lk, ll, _, _ = c2.keys(np.arange(0, 20000, 211))
        got = sh.scan(d(lk), d(ll), 300)
        exp = o.scan(lk, ll, 300, maxV=MAXV)
        for x, y, name in zip(got, exp, ["counts", "values", "value lengths", "keys", "key lengths"]):
            np.testing.assert_array_equal(x.cpu().numpy(), y, err_msg=name)
    finally:
        g.close()
        dist.destroy_process_group()
