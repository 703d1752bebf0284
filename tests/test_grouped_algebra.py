"""The state algebra of the grouped batched form (mt_grouped.cu), restated on
the host: a request's transfer function maps the key's state before it
(absent / present with the value the tree held / present with the value of
request x) to the state after it; a run's functions compose associatively, and
applying the exclusive prefix to the key's initial state gives every request
the state it would see if the run were served one request after the other.
Checked here against that one-by-one service on random runs, with random
bracketings of the composition (a parallel scan may group them any way)."""
import numpy as np

ABSENT, KEEP = -2, -1  # kGAbsent, kGKeep; any value >= 0 is the id of the write the key holds
INSERT, ERASE, FIND, UPDATE = 0, 1, 2, 3  # MT_REQ_*


def apply(s, f):
    a, p = f
    if s == ABSENT:
        return a
    return s if p == KEEP else p


def compose(f, g):  # f, then g
    return (apply(f[0], g), apply(f[1], g))


IDENTITY = (ABSENT, KEEP)


def fn(kind, rid):
    return {FIND: IDENTITY, INSERT: (rid, KEEP), UPDATE: (ABSENT, rid), ERASE: (ABSENT, ABSENT)}[kind]


def serve_one_by_one(init_present, kinds):
    """(state before each request, results, final state) by plain sequential service."""
    s = KEEP if init_present else ABSENT
    before, results = [], []
    for rid, k in enumerate(kinds):
        before.append(s)
        if k == INSERT:
            results.append(s == ABSENT)
            if s == ABSENT:
                s = rid
        elif k == UPDATE:
            results.append(s != ABSENT)
            if s != ABSENT:
                s = rid
        elif k == ERASE:
            results.append(s != ABSENT)
            s = ABSENT
        else:
            results.append(None)
    return before, results, s


def fold(fs, rng):
    """Compose fs (in order) under a random bracketing."""
    if not fs:
        return IDENTITY
    if len(fs) == 1:
        return fs[0]
    cut = int(rng.integers(1, len(fs)))
    return compose(fold(fs[:cut], rng), fold(fs[cut:], rng))


def test_scanned_states_equal_one_by_one_service():
    rng = np.random.default_rng(12)
    for _ in range(3000):
        n = int(rng.integers(1, 12))
        kinds = rng.integers(0, 4, n).tolist()
        init_present = bool(rng.integers(0, 2))
        before, results, final = serve_one_by_one(init_present, kinds)
        fs = [fn(k, rid) for rid, k in enumerate(kinds)]
        s0 = KEEP if init_present else ABSENT
        for j in range(n):
            pre = fold(fs[:j], rng)
            sb = apply(s0, pre)
            assert sb == before[j], (kinds, init_present, j)
            if kinds[j] == INSERT:
                assert (sb == ABSENT) == results[j]
            elif kinds[j] in (UPDATE, ERASE):
                assert (sb != ABSENT) == results[j]
        assert apply(s0, fold(fs, rng)) == final


def test_composition_is_associative_and_identity_is_neutral():
    # Every function a run can produce: from "absent" to absent or a write, from
    # "present" to kept, absent or a write (never "kept" from absent: there is
    # no value to keep).
    rng = np.random.default_rng(13)
    ids = [0, 1, 2, 3]
    fns = [(a, p) for a in [ABSENT] + ids for p in [KEEP, ABSENT] + ids]
    for _ in range(5000):
        f, g, h = (fns[int(i)] for i in rng.integers(0, len(fns), 3))
        assert compose(compose(f, g), h) == compose(f, compose(g, h))
        assert compose(IDENTITY, f) == f == compose(f, IDENTITY)
        assert compose(f, g)[0] != KEEP  # closed: compositions stay in the domain
