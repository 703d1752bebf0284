"""Uniform numpy-in / numpy-out adapters over the three index implementations
the tests compare: the CUDA library under test (GpuIndex) and the CPU oracle
(OracleIndex).

keys are 2-D uint32 arrays (n, max_key_length); values (n, max_value_length).
"""
import numpy as np

from oracle.pyoracle import CpuOracle


def _u32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint32)


class OracleIndex:
    name = "oracle"

    def __init__(self, shards=1, threads=1):
        self.o = CpuOracle(shards, threads)

    def insert(self, keys, klens, vals, vlens, n=None, upsert=False):
        keys, vals = _u32(keys), _u32(vals)
        n = len(keys) if n is None else n
        res = np.zeros(n, np.uint8)
        self.o.insert(keys, keys.shape[1], _u32(klens), vals, vals.shape[1], _u32(vlens), n, res, upsert)
        return res

    def update(self, keys, klens, vals, vlens, n=None):
        keys, vals = _u32(keys), _u32(vals)
        n = len(keys) if n is None else n
        res = np.zeros(n, np.uint8)
        self.o.update(keys, keys.shape[1], _u32(klens), vals, vals.shape[1], _u32(vlens), n, res)
        return res

    def erase(self, keys, klens, n=None):
        keys = _u32(keys)
        n = len(keys) if n is None else n
        res = np.zeros(n, np.uint8)
        self.o.erase(keys, keys.shape[1], _u32(klens), n, res)
        return res

    def find(self, keys, klens, maxV, n=None):
        keys = _u32(keys)
        n = len(keys) if n is None else n
        vals = np.zeros((n, maxV), np.uint32)
        vlens = np.zeros(n, np.uint32)
        self.o.find(keys, keys.shape[1], _u32(klens), vals, maxV, vlens, n)
        return vals, vlens

    def mixed(self, types, keys, klens, vals, vlens, n=None):
        keys = _u32(keys)
        vals = _u32(vals).copy()
        vlens = _u32(vlens).copy()
        n = len(keys) if n is None else n
        res = np.zeros(n, np.uint8)
        self.o.mixed(np.ascontiguousarray(types, np.uint8), keys, keys.shape[1], _u32(klens), vals, vals.shape[1],
                     vlens, res, n)
        return vals, vlens, res

    def scan(self, lower, lower_lens, max_count, upper=None, upper_lens=None, maxV=1, nq=None):
        lower = _u32(lower)
        nq = len(lower) if nq is None else nq
        maxK = lower.shape[1]
        counts = np.zeros(nq, np.uint32)
        vals = np.zeros((nq, max_count, maxV), np.uint32)
        vlens = np.zeros((nq, max_count), np.uint32)
        okeys = np.zeros((nq, max_count, maxK), np.uint32)
        oklens = np.zeros((nq, max_count), np.uint32)
        self.o.scan(lower, _u32(lower_lens), maxK, max_count, nq, None if upper is None else _u32(upper),
                    None if upper_lens is None else _u32(upper_lens), upper is not None, counts, vals, maxV, vlens,
                    okeys, oklens)
        return counts, vals, vlens, okeys, oklens

    def dump(self, maxK, maxV):
        return self.o.dump(maxK, maxV)


class _TorchIndex:
    """Device-buffer plumbing."""

    def __init__(self):
        import torch
        self.torch = torch

    def d(self, a, dtype=None):
        if a is None:
            return None
        t = self.torch.from_numpy(np.ascontiguousarray(a))
        return t.cuda()

    def zeros(self, shape, dtype):
        return self.torch.zeros(shape, dtype=dtype, device="cuda")

    @staticmethod
    def h(t):
        return t.cpu().numpy()


class GpuIndex(_TorchIndex):
    name = "b200"

    def __init__(self, tile_size=8, pool_bytes=1 << 30):
        super().__init__()
        from indexingpu_b200 import GpuMasstree
        self.t = GpuMasstree(tile_size=tile_size, pool_bytes=pool_bytes)

    def close(self):
        self.t.close()

    def insert(self, keys, klens, vals, vlens, n=None, upsert=False):
        torch = self.torch
        keys, vals = _u32(keys), _u32(vals)
        n = len(keys) if n is None else n
        res = self.zeros(n, torch.bool)
        self.t.insert(self.d(keys), keys.shape[1], self.d(_u32(klens)), self.d(vals), vals.shape[1],
                      self.d(_u32(vlens)), n, update_if_exists=upsert, results=res)
        self.t.sync()
        return self.h(res).astype(np.uint8)

    def update(self, keys, klens, vals, vlens, n=None):
        torch = self.torch
        keys, vals = _u32(keys), _u32(vals)
        n = len(keys) if n is None else n
        res = self.zeros(n, torch.bool)
        self.t.update(self.d(keys), keys.shape[1], self.d(_u32(klens)), self.d(vals), vals.shape[1],
                      self.d(_u32(vlens)), n, results=res)
        self.t.sync()
        return self.h(res).astype(np.uint8)

    def erase(self, keys, klens, n=None, merge=False, remove_empty_layers=False):
        torch = self.torch
        keys = _u32(keys)
        n = len(keys) if n is None else n
        res = self.zeros(n, torch.bool)
        self.t.erase(self.d(keys), keys.shape[1], self.d(_u32(klens)), n, results=res, merge=merge,
                     remove_empty_layers=remove_empty_layers)
        self.t.sync()
        return self.h(res).astype(np.uint8)

    def find(self, keys, klens, maxV, n=None, concurrent=False):
        torch = self.torch
        keys = _u32(keys)
        n = len(keys) if n is None else n
        vals = self.zeros((n, maxV), torch.uint32)
        vlens = self.zeros(n, torch.uint32)
        self.t.find(self.d(keys), keys.shape[1], self.d(_u32(klens)), vals, maxV, vlens, n, concurrent=concurrent)
        self.t.sync()
        return self.h(vals), self.h(vlens)

    def mixed(self, types, keys, klens, vals, vlens, n=None, bucket_keys=False, merge=False,
              remove_empty_layers=False):
        torch = self.torch
        keys = _u32(keys)
        n = len(keys) if n is None else n
        dv = self.d(_u32(vals))
        dvl = self.d(_u32(vlens))
        res = self.zeros(n, torch.bool)
        self.t.mixed_batch(self.d(np.ascontiguousarray(types, np.uint8)), self.d(keys), keys.shape[1],
                           self.d(_u32(klens)), dv, dv.shape[1], dvl, res, n, bucket_keys=bucket_keys, merge=merge,
                           remove_empty_layers=remove_empty_layers)
        self.t.sync()
        return self.h(dv), self.h(dvl), self.h(res).astype(np.uint8)

    def scan(self, lower, lower_lens, max_count, upper=None, upper_lens=None, maxV=1, nq=None, concurrent=False):
        torch = self.torch
        lower = _u32(lower)
        nq = len(lower) if nq is None else nq
        maxK = lower.shape[1]
        counts = self.zeros(nq, torch.uint32)
        vals = self.zeros((nq, max_count, maxV), torch.uint32)
        vlens = self.zeros((nq, max_count), torch.uint32)
        okeys = self.zeros((nq, max_count, maxK), torch.uint32)
        oklens = self.zeros((nq, max_count), torch.uint32)
        self.t.scan(self.d(lower), self.d(_u32(lower_lens)), maxK, max_count, nq,
                    None if upper is None else self.d(_u32(upper)),
                    None if upper_lens is None else self.d(_u32(upper_lens)), counts, vals, maxV, vlens, okeys,
                    oklens, concurrent=concurrent)
        self.t.sync()
        return self.h(counts), self.h(vals), self.h(vlens), self.h(okeys), self.h(oklens)


def dump_by_scan(g, maxK, maxV, n):
    """Every (key, key length, value, value length) of a GpuIndex in key order,
    by one scan from the smallest key."""
    import torch
    t = g.t
    lower = torch.zeros((1, maxK), dtype=torch.uint32, device="cuda")
    lens = torch.ones(1, dtype=torch.uint32, device="cuda")
    counts = torch.zeros(1, dtype=torch.uint32, device="cuda")
    vals = torch.zeros((1, n, maxV), dtype=torch.uint32, device="cuda")
    vlens = torch.zeros((1, n), dtype=torch.uint32, device="cuda")
    keys = torch.zeros((1, n, maxK), dtype=torch.uint32, device="cuda")
    klens = torch.zeros((1, n), dtype=torch.uint32, device="cuda")
    t.scan(lower, lens, maxK, n, 1, counts=counts, values=vals, max_value_length=maxV, value_lengths=vlens,
           out_keys=keys, out_key_lengths=klens)
    t.sync()
    c = int(counts[0])
    return [x[0, :c].cpu().numpy() for x in (keys, klens, vals, vlens)]


def same_state(g, o, maxK, maxV):
    """The GpuIndex holds exactly the oracle's keys and values."""
    n = o.o.size()
    a = dump_by_scan(g, maxK, maxV, n + 8)
    b = o.dump(maxK, maxV)
    assert len(a[0]) == n
    for x, y, name in zip(a, b, ["keys", "key lengths", "values", "value lengths"]):
        np.testing.assert_array_equal(x, y, err_msg=name)
