"""Regenerate tests/golden/unittest_inputs_*.npz.

Compiles gen_unittest_inputs.cpp with g++ (libstdc++'s std::mt19937 and
std::uniform_int_distribution, as the reference's test uses) and packs the
inputs of the four shapes the reference instantiates
(test/unittest_masstree.cu:755-758) at its default of 1024 keys (:764).
Run: python tests/golden/make_unittest_inputs.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPES = [(1, 1, 1, 1), (1, 200, 1, 1), (1, 1, 1, 200), (1, 200, 1, 200)]
NUM_KEYS = 1024


def shape_name(s):
    return f"k{s[0]}-{s[1]}_v{s[2]}-{s[3]}"


def main():
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "gen")
        subprocess.check_call(["g++", "-O2", "-std=c++17", os.path.join(HERE, "gen_unittest_inputs.cpp"), "-o", exe])
        for s in SHAPES:
            out = os.path.join(td, "o.bin")
            subprocess.check_call([exe, str(NUM_KEYS), *map(str, s), out])
            raw = np.fromfile(out, dtype=np.uint32)
            n, maxK, maxV = NUM_KEYS, s[1], s[3]
            parts, off = {}, 0
            for name, size in [("keys", n * maxK), ("lengths", n), ("values", n * maxV), ("value_lengths", n),
                               ("values2", n * maxV), ("keys_not_exist", n * maxK),
                               ("shuffle_order", n), ("mix_order", 10 * (n // 4))]:
                parts[name] = raw[off:off + size]
                off += size
            assert off == raw.size
            parts["keys"] = parts["keys"].reshape(n, maxK)
            parts["keys_not_exist"] = parts["keys_not_exist"].reshape(n, maxK)
            parts["values"] = parts["values"].reshape(n, maxV)
            parts["values2"] = parts["values2"].reshape(n, maxV)
            np.savez_compressed(os.path.join(HERE, f"unittest_inputs_{shape_name(s)}.npz"),
                                shape=np.array(s, dtype=np.uint32), **parts)
            print("wrote", shape_name(s))


if __name__ == "__main__":
    main()
