"""mt_mixed_batches with MT_FLAG_GROUP_BY_KEY (every sub-batch served at once,
each key's requests resolved in sub-batch order) against one mt_mixed_batch
call per sub-batch on an identical tree: per-request results, find outputs and
the final contents must match exactly.  Each sub-batch touches a key at most
once (so one call per sub-batch has one outcome); keys come back across
sub-batches: hot keys of a Zipf draw, and keys erased, inserted again, updated
and found in later sub-batches.  With fewer hash bits, different keys share
hashes and those runs are served one by one."""
import numpy as np
import pytest

from indexingpu_b200 import workload as wl
from indexingpu_b200.masstree import pack_subbatches
from test_gpu_batches import MAXK, MAXV, _check_outputs, _compare, _dev, _dump, _make_pair, _touch_once

pytestmark = pytest.mark.gpu
N_PRE = 20000


def _made(c2, types, ids, salt):
    """A sub-batch of the given kinds on the given key ids; inserts and updates
    carry values derived from the key and `salt`."""
    keys, lens, vals, vlens = c2.keys(np.asarray(ids))
    types = np.asarray(types, np.uint8)
    with np.errstate(over="ignore"):
        vals = (vals.astype(np.uint64) * np.uint64(2654435761) + np.uint64(salt)).astype(np.uint32)
    write = (types == wl.REQ_INSERT) | (types == wl.REQ_UPDATE)
    vals = np.where(write[:, None] & (np.arange(MAXV)[None, :] < vlens[:, None]), vals, 0).astype(np.uint32)
    vlens = np.where(types == wl.REQ_FIND, 0, vlens).astype(np.uint32)
    return dict(types=types, ids=np.asarray(ids), keys=keys, lens=lens, vals=vals, vlens=vlens)


def _plan(c2):
    rng = np.random.default_rng(41)
    bts = [_touch_once(c2.batch(b, n)) for b, n in enumerate([4000, 300, 2500, 1, 5000])]
    # Keys erased, then inserted again, found, updated, found, erased, found.
    e = rng.choice(N_PRE, 400, replace=False)
    seq = [wl.REQ_ERASE, wl.REQ_FIND, wl.REQ_INSERT, wl.REQ_FIND, wl.REQ_UPDATE, wl.REQ_UPDATE, wl.REQ_FIND,
           wl.REQ_ERASE, wl.REQ_FIND, wl.REQ_INSERT]
    for k, kind in enumerate(seq):
        bts.append(_made(c2, np.full(len(e), kind), e, 100 + k))
        bts.append(_touch_once(c2.batch(20 + k, 700)))
    # Fresh keys inserted, then updated and found in the same list.
    f = N_PRE + (1 << 28) + np.arange(300)
    bts.append(_made(c2, np.full(300, wl.REQ_INSERT), f, 7))
    bts.append(_made(c2, np.full(300, wl.REQ_FIND), f, 0))
    bts.append(_made(c2, np.full(300, wl.REQ_UPDATE), f, 8))
    bts.append(_made(c2, np.where(np.arange(300) % 2 == 0, wl.REQ_ERASE, wl.REQ_FIND), f, 0))
    return bts


@pytest.mark.parametrize("tf,tw,bits", [(8, 32, 64), (4, 16, 64), (8, 32, 12), (8, 32, 3)])
def test_grouped_matches_per_call(tf, tw, bits):
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    ref, new = _make_pair(torch, c2, N_PRE, tf, tw)
    try:
        bts = _plan(c2)
        ref_sbs = [_dev(torch, bt) for bt in bts]
        new_sbs = [_dev(torch, bt) for bt in bts]
        for sb in ref_sbs:
            ref.mixed_batch(sb["types"], sb["keys"], MAXK, sb["lens"], sb["vals"], MAXV, sb["vlens"], sb["results"],
                            sb["n"])
        ref.sync()
        new.set_group_hash_bits(bits)
        desc = torch.from_numpy(pack_subbatches(new_sbs)).cuda()
        new.reserve_batches(len(new_sbs), sum(sb["n"] for sb in new_sbs))
        new.mixed_batches(desc, len(new_sbs), MAXK, MAXV, group_by_key=True)
        new.sync()
        for r, s, bt in zip(ref_sbs, new_sbs, bts):
            _check_outputs(r, s, bt)
        _compare(_dump(torch, ref, 80000), _dump(torch, new, 80000))
        ok, _, msg = new.validate()
        assert ok, msg
    finally:
        ref.close()
        new.close()


def test_grouped_twice_and_after_other_forms():
    """Two grouped calls in a row (the second on the first's outcome, scratch
    reused), then a forked call, all against one call per sub-batch."""
    import torch
    c2 = wl.C2(n_preload=N_PRE, n_prefixes=64)
    ref, new = _make_pair(torch, c2, N_PRE, 8, 32)
    try:
        plans = [[_touch_once(c2.batch(50 + 10 * r + b, n)) for b, n in enumerate([3000, 900, 2000])]
                 for r in range(3)]
        new.reserve_batches(3, 6000)
        for r, plan in enumerate(plans):
            ref_sbs = [_dev(torch, bt) for bt in plan]
            new_sbs = [_dev(torch, bt) for bt in plan]
            for sb in ref_sbs:
                ref.mixed_batch(sb["types"], sb["keys"], MAXK, sb["lens"], sb["vals"], MAXV, sb["vlens"],
                                sb["results"], sb["n"])
            ref.sync()
            desc = torch.from_numpy(pack_subbatches(new_sbs)).cuda()
            new.mixed_batches(desc, len(new_sbs), MAXK, MAXV, group_by_key=r < 2)
            new.sync()
            for a, b, bt in zip(ref_sbs, new_sbs, plan):
                _check_outputs(a, b, bt)
        _compare(_dump(torch, ref, 80000), _dump(torch, new, 80000))
        ok, _, msg = new.validate()
        assert ok, msg
    finally:
        ref.close()
        new.close()
