"""TEST INFRASTRUCTURE ONLY.  ctypes bindings of the two oracles.

CpuOracle   -- oracle/build/libmt_oracle.so, the CPU restatement (mt_oracle.cpp)
RefMasstree -- oracle/_ref/libref_masstree.so, the reference's own gpu_masstree
               compiled from its headers (ref_capi.cu); runs on the GPU.
Arrays for CpuOracle are numpy; RefMasstree takes device pointers (ints).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPU_LIB = os.path.join(HERE, "build", "libmt_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_masstree.so")

_p = ctypes.c_void_p
_u32 = ctypes.c_uint32
_int = ctypes.c_int


def build_cpu():
    if not os.path.exists(CPU_LIB) or os.path.getmtime(CPU_LIB) < os.path.getmtime(os.path.join(HERE, "mt_oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    return CPU_LIB


def _np(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_p)


class CpuOracle:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(build_cpu())
            sig = {
                "oracle_create": (_p, [_u32]),
                "oracle_destroy": (None, [_p]),
                "oracle_size": (ctypes.c_uint64, [_p]),
                "oracle_insert": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p, _int, _u32]),
                "oracle_update": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p, _u32]),
                "oracle_erase": (None, [_p, _p, _u32, _p, _u32, _p, _u32]),
                "oracle_find": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _u32]),
                "oracle_mixed": (None, [_p, _p, _p, _u32, _p, _p, _u32, _p, _p, _u32, _u32]),
                "oracle_scan": (None, [_p, _p, _p, _u32, _u32, _u32, _p, _p, _int, _p, _p, _u32, _p, _p, _p]),
                "oracle_dump": (None, [_p, _p, _u32, _p, _p, _u32, _p]),
            }
            for k, (r, a) in sig.items():
                f = getattr(lib, k)
                f.restype = r
                f.argtypes = a
            cls._lib = lib
        return cls._lib

    def __init__(self, shards=1, threads=1):
        self.L = self.lib()
        self.h = self.L.oracle_create(shards)
        self.threads = threads

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def size(self):
        return int(self.L.oracle_size(self.h))

    def insert(self, keys, maxK, klens, vals, maxV, vlens, n, results=None, upsert=False):
        self.L.oracle_insert(self.h, _np(keys), maxK, _np(klens), _np(vals), maxV, _np(vlens), n, _np(results),
                             int(upsert), self.threads)

    def update(self, keys, maxK, klens, vals, maxV, vlens, n, results=None):
        self.L.oracle_update(self.h, _np(keys), maxK, _np(klens), _np(vals), maxV, _np(vlens), n, _np(results),
                             self.threads)

    def erase(self, keys, maxK, klens, n, results=None):
        self.L.oracle_erase(self.h, _np(keys), maxK, _np(klens), n, _np(results), self.threads)

    def find(self, keys, maxK, klens, vals, maxV, vlens, n):
        self.L.oracle_find(self.h, _np(keys), maxK, _np(klens), _np(vals), maxV, _np(vlens), n, self.threads)

    def mixed(self, kinds, keys, maxK, klens, vals, maxV, vlens, results, n):
        self.L.oracle_mixed(self.h, _np(kinds), _np(keys), maxK, _np(klens), _np(vals), maxV, _np(vlens),
                            _np(results), n, self.threads)

    def scan(self, lower, lower_lens, maxK, max_count, nq, upper=None, upper_lens=None, use_upper=False,
             counts=None, vals=None, maxV=1, vlens=None, out_keys=None, out_klens=None):
        self.L.oracle_scan(self.h, _np(lower), _np(lower_lens), maxK, max_count, nq, _np(upper), _np(upper_lens),
                           int(use_upper), _np(counts), _np(vals), maxV, _np(vlens), _np(out_keys), _np(out_klens))

    def dump(self, maxK, maxV):
        n = self.size()
        keys = np.zeros((n, maxK), np.uint32)
        klens = np.zeros(n, np.uint32)
        vals = np.zeros((n, maxV), np.uint32)
        vlens = np.zeros(n, np.uint32)
        self.L.oracle_dump(self.h, _np(keys), maxK, _np(klens), _np(vals), maxV, _np(vlens))
        return keys, klens, vals, vlens


class RefMasstree:
    """The reference's gpu_masstree (tile 16, adapter defaults) over device pointers."""
    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(REF_LIB)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_LIB):
                raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference is present")
            lib = ctypes.CDLL(REF_LIB)
            sig = {
                "ref_create": (_p, [ctypes.c_float]),
                "ref_destroy": (None, [_p]),
                "ref_insert": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p]),
                "ref_update": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p]),
                "ref_erase": (None, [_p, _p, _u32, _p, _u32, _p]),
                "ref_find": (None, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _int, _p]),
                "ref_mixed": (None, [_p, _p, _p, _u32, _p, _p, _u32, _p, _p, _u32, _p]),
                "ref_scan": (None, [_p, _p, _p, _u32, _u32, _u32, _p, _p, _int, _p, _p, _u32, _p, _p, _p, _p]),
                "ref_sync": (_int, [_p]),
            }
            for k, (r, a) in sig.items():
                f = getattr(lib, k)
                f.restype = r
                f.argtypes = a
            cls._lib = lib
        return cls._lib

    def __init__(self, pool_ratio):
        self.L = self.lib()
        self.h = self.L.ref_create(pool_ratio)

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _d(t):
        return None if t is None else t.data_ptr()

    def insert(self, keys, maxK, klens, vals, maxV, vlens, n, stream=None):
        d = self._d
        self.L.ref_insert(self.h, d(keys), maxK, d(klens), d(vals), maxV, d(vlens), n, stream)

    def update(self, keys, maxK, klens, vals, maxV, vlens, n, stream=None):
        d = self._d
        self.L.ref_update(self.h, d(keys), maxK, d(klens), d(vals), maxV, d(vlens), n, stream)

    def erase(self, keys, maxK, klens, n, stream=None):
        d = self._d
        self.L.ref_erase(self.h, d(keys), maxK, d(klens), n, stream)

    def find(self, keys, maxK, klens, vals, maxV, vlens, n, concurrent=False, stream=None):
        d = self._d
        self.L.ref_find(self.h, d(keys), maxK, d(klens), d(vals), maxV, d(vlens), n, int(concurrent), stream)

    def mixed(self, types, keys, maxK, klens, vals, maxV, vlens, results, n, stream=None):
        d = self._d
        self.L.ref_mixed(self.h, d(types), d(keys), maxK, d(klens), d(vals), maxV, d(vlens), d(results), n, stream)

    def scan(self, lower, lower_lens, maxK, max_count, nq, upper=None, upper_lens=None, use_upper=False, counts=None,
             vals=None, maxV=1, vlens=None, out_keys=None, out_klens=None, stream=None):
        d = self._d
        self.L.ref_scan(self.h, d(lower), d(lower_lens), maxK, max_count, nq, d(upper), d(upper_lens), int(use_upper),
                        d(counts), d(vals), maxV, d(vlens), d(out_keys), d(out_klens), stream)

    def sync(self, stream=None):
        rc = self.L.ref_sync(stream)
        if rc != 0:
            raise RuntimeError(f"reference gpu_masstree CUDA error {rc}")
