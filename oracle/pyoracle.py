"""TEST INFRASTRUCTURE ONLY.  ctypes binding of the CPU oracle
(oracle/build/libmt_oracle.so, the restatement in mt_oracle.cpp).  Arrays are
numpy.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPU_LIB = os.path.join(HERE, "build", "libmt_oracle.so")

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
