"""The device API (include/mt/device.cuh) called from user kernels.

tests/cpp/device_api_check.cu holds kernels written the way the reference's
README shows its device-side API (README.md:114-166): a cooperative_groups
tile per request, an allocator context from index.allocator_, a reclaimer
context from index.reclaimer_.  They insert, find (plain and concurrent),
update, erase, scan (with and without an upper bound) and, in one fused kernel,
insert then find.  Every result is compared with the oracle, and the tree they
leave must hold the oracle's contents and pass the structural check.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from indexes import OracleIndex, same_state
from indexingpu_b200 import workload as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
LIB = os.path.join(CPP, "build", "libmt_device_check.so")

_p, _u32, _int = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
SIGS = {
    "dev_find": [_p, _u32, _p, _u32, _p, _p, _u32, _p, _u32, _int, _p],
    "dev_write": [_p, _u32, _int, _p, _u32, _p, _p, _u32, _p, _u32, _p, _p],
    "dev_insert_then_find": [_p, _u32, _p, _u32, _p, _p, _u32, _p, _u32, _p, _p, _p],
    "dev_scan": [_p, _u32, _p, _p, _u32, _u32, _u32, _p, _p, _int, _p, _p, _u32, _p, _p, _p, _p],
}


def load_check_lib():
    subprocess.check_call(["make", "-s", "-C", CPP])
    from indexingpu_b200 import _lib
    _lib.load()  # libmt_b200.so first (the check library links against it)
    lib = ctypes.CDLL(LIB)
    for k, a in SIGS.items():
        getattr(lib, k).argtypes = a
        getattr(lib, k).restype = _int
    return lib


def test_check_library_builds_and_exports():
    lib = load_check_lib()
    for k in SIGS:
        assert hasattr(lib, k)


def _d(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class DeviceApiIndex:
    """numpy in / numpy out over the user kernels."""

    def __init__(self, lib, tree, tile):
        import torch
        self.torch, self.lib, self.tree, self.tile = torch, lib, tree, tile

    def write(self, kind, keys, lens, vals=None, vlens=None):
        torch = self.torch
        n = len(keys)
        res = torch.zeros(n, dtype=torch.uint8, device="cuda")
        dk, dl = _d(torch, keys), _d(torch, lens)
        dv = None if vals is None else _d(torch, vals)
        dvl = None if vlens is None else _d(torch, vlens)
        rc = self.lib.dev_write(self.tree._h, self.tile, kind, _ptr(dk), keys.shape[1], _ptr(dl), _ptr(dv),
                                0 if vals is None else vals.shape[1], _ptr(dvl), n, _ptr(res), None)
        assert rc == 0
        self.tree.sync()
        return res.cpu().numpy()

    def find(self, keys, lens, maxV, concurrent):
        torch = self.torch
        n = len(keys)
        vals = torch.zeros((n, maxV), dtype=torch.uint32, device="cuda")
        vlens = torch.zeros(n, dtype=torch.uint32, device="cuda")
        dk, dl = _d(torch, keys), _d(torch, lens)
        rc = self.lib.dev_find(self.tree._h, self.tile, _ptr(dk), keys.shape[1], _ptr(dl), _ptr(vals), maxV,
                               _ptr(vlens), n, 1 if concurrent else 0, None)
        assert rc == 0
        self.tree.sync()
        return vals.cpu().numpy(), vlens.cpu().numpy()

    def insert_then_find(self, keys, lens, vals, vlens):
        torch = self.torch
        n = len(keys)
        res = torch.zeros(n, dtype=torch.uint8, device="cuda")
        found = torch.zeros(n, dtype=torch.uint32, device="cuda")
        dk, dl, dv, dvl = (_d(torch, a) for a in (keys, lens, vals, vlens))
        rc = self.lib.dev_insert_then_find(self.tree._h, self.tile, _ptr(dk), keys.shape[1], _ptr(dl), _ptr(dv),
                                           vals.shape[1], _ptr(dvl), n, _ptr(res), _ptr(found), None)
        assert rc == 0
        self.tree.sync()
        return res.cpu().numpy(), found.cpu().numpy()

    def scan(self, lower, lower_lens, max_count, maxV, upper=None, upper_lens=None):
        torch = self.torch
        nq, maxK = lower.shape
        z = lambda *s: torch.zeros(s, dtype=torch.uint32, device="cuda")  # noqa: E731
        counts, vals, vlens, okeys, oklens = z(nq), z(nq, max_count, maxV), z(nq, max_count), \
            z(nq, max_count, maxK), z(nq, max_count)
        dlo, dll = _d(torch, lower), _d(torch, lower_lens)
        dup = None if upper is None else _d(torch, upper)
        dul = None if upper is None else _d(torch, upper_lens)
        rc = self.lib.dev_scan(self.tree._h, self.tile, _ptr(dlo), _ptr(dll), maxK, max_count, nq, _ptr(dup),
                               _ptr(dul), 0 if upper is None else 1, _ptr(counts), _ptr(vals), maxV, _ptr(vlens),
                               _ptr(okeys), _ptr(oklens), None)
        assert rc == 0
        self.tree.sync()
        return tuple(x.cpu().numpy() for x in (counts, vals, vlens, okeys, oklens))


def _assert_found(gv, gl, ov, ol, what):
    np.testing.assert_array_equal(gl, ol, err_msg=f"{what}: value lengths")
    live = np.arange(ov.shape[1])[None, :] < np.minimum(ol, ov.shape[1])[:, None]
    assert not ((gv != ov) & live).any(), f"{what}: values"


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [8, 16, 32])
def test_user_kernels_match_oracle(tile):
    import torch  # noqa: F401

    from indexes import GpuIndex
    lib = load_check_lib()
    c2 = wl.C2(n_preload=20000, n_prefixes=64)
    keys, lens, vals, vlens = c2.keys(np.arange(20000))
    g, o = GpuIndex(tile_size=tile, pool_bytes=256 << 20), OracleIndex()
    dev = DeviceApiIndex(lib, g.t, tile)
    try:
        # Inserts (half the keys twice: the second time they must fail).
        np.testing.assert_array_equal(dev.write(0, keys, lens, vals, vlens), o.insert(keys, lens, vals, vlens))
        np.testing.assert_array_equal(dev.write(0, keys[:10000], lens[:10000], vals[:10000], vlens[:10000]),
                                      o.insert(keys[:10000], lens[:10000], vals[:10000], vlens[:10000]))
        # Finds: present keys and absent ones, plain and concurrent.
        fk = np.concatenate([keys[::3], c2.keys(np.arange(20000, 23000))[0]])
        fl = np.concatenate([lens[::3], c2.keys(np.arange(20000, 23000))[1]])
        ov, ol = o.find(fk, fl, 8)
        for conc in (False, True):
            gv, gl = dev.find(fk, fl, 8, conc)
            _assert_found(gv, gl, ov, ol, f"find concurrent={conc}")
        # Updates (some of absent keys), upserts, erases.
        uk = np.concatenate([keys[:4000], fk[-500:]])
        ul = np.concatenate([lens[:4000], fl[-500:]])
        uv = np.concatenate([vals[:4000] ^ np.uint32(0x1234567), vals[:500]])
        uvl = np.concatenate([(vlens[:4000] % 8) + 1, vlens[:500]]).astype(np.uint32)
        np.testing.assert_array_equal(dev.write(2, uk, ul, uv, uvl), o.update(uk, ul, uv, uvl))
        np.testing.assert_array_equal(dev.write(1, uk[::2], ul[::2], uv[::2] + 1, uvl[::2]),
                                      o.insert(uk[::2], ul[::2], uv[::2] + 1, uvl[::2], upsert=True))
        ek = np.concatenate([keys[5000:9000], fk[-300:]])
        el = np.concatenate([lens[5000:9000], fl[-300:]])
        np.testing.assert_array_equal(dev.write(3, ek, el), o.erase(ek, el))
        # Insert then find in one kernel (fresh keys: every insert succeeds and
        # every key is found right after its insert).
        nk, nl, nv, nvl = c2.keys(np.arange(30000, 34000))
        res, found = dev.insert_then_find(nk, nl, nv, nvl)
        np.testing.assert_array_equal(res, o.insert(nk, nl, nv, nvl))
        np.testing.assert_array_equal(found, nvl)
        # Scans from present and absent lower bounds, with and without upper bounds.
        lo_k, lo_l = fk[::7], fl[::7]
        up_k = np.zeros_like(lo_k)
        up_k[:, 0] = lo_k[:, 0] + np.uint32(1 << 24)
        up_l = np.ones(len(lo_k), np.uint32)
        a = dev.scan(lo_k, lo_l, 40, 8)
        b = o.scan(lo_k, lo_l, 40, maxV=8)
        for x, y, name in zip(a, b, ["counts", "values", "value lengths", "keys", "key lengths"]):
            np.testing.assert_array_equal(x, y, err_msg=f"scan: {name}")
        a = dev.scan(lo_k, lo_l, 40, 8, up_k, up_l)
        b = o.scan(lo_k, lo_l, 40, up_k, up_l, maxV=8)
        for x, y, name in zip(a, b, ["counts", "values", "value lengths", "keys", "key lengths"]):
            np.testing.assert_array_equal(x, y, err_msg=f"scan with upper bound: {name}")
        # The host API sees what the user kernels left, and the tree is sound.
        g.t.reclaim()
        same_state(g, o, c2.maxK, c2.maxV)
        ok, nkeys, msg = g.t.validate()
        assert ok and nkeys == o.o.size(), msg
    finally:
        g.close()
