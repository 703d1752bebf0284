"""Autotuner for the batched form (mt_mixed_batches).

Searches the form and launch shape of the call over
  form (three class kernels per sub-batch on forked streams, one persistent
  launch for all sub-batches, or all sub-batches at once grouped by key) x
  find tile (lanes per find: 4, 8, 16, 32) x write tile (lanes per insert,
  update and erase: 16, 32) x key-length bucketing (off, on; the grouped
  form has no buckets and runs once per tile pair),
then, for the best of those, blocks per SM 1..8.  This is coordinate descent
(40 + 8 trials rather than the 384 points of the full grid): blocks per SM
only trades occupancy against per-warp registers, and is measured with the
other choices fixed.

Every trial runs on a fresh case from `make_case(i)`: the tree changes under
every trial (inserts add keys, erases remove them), so replaying one case would
turn later trials' inserts into cheap "already present" misses.  The cases must
have the same shape (sub-batch sizes and mix) for the comparison to be fair.
"""
import time

FIND_TILES = (4, 8, 16, 32)
WRITE_TILES = (16, 32)
BUCKETING = (False, True)
FORMS = ("forked", "persistent", "grouped")
BLOCKS_PER_SM = tuple(range(1, 9))


def apply(tree, config):
    """Set a tree's launch shape to `config` (a dict from tune())."""
    tree.set_tile_size(config["find_tile"])
    tree.set_write_tile_size(config["write_tile"])
    tree.set_blocks_per_sm(config["blocks_per_sm"])


def time_trial(tree, case, config, stream):
    """Run one case under one configuration; returns Mops/s (device time)."""
    import torch
    apply(tree, config)
    tree.reserve_batches(case["num_subbatches"], case["total"])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tree.mixed_batches(case["descriptors"], case["num_subbatches"], case["max_key_length"],
                       case["max_value_length"], stream=stream, bucket_keys=config["bucketing"],
                       persistent=config.get("form") == "persistent", group_by_key=config.get("form") == "grouped")
    e1.record(stream)
    tree.sync(stream)
    return case["total"] / (e0.elapsed_time(e1) / 1e3) / 1e6


def tune(tree, make_case, stream=None, find_tiles=FIND_TILES, write_tiles=WRITE_TILES, bucketing=BUCKETING,
         blocks_per_sm=BLOCKS_PER_SM, log=None, trial=time_trial, forms=FORMS):
    """Coordinate-descent search; returns (best config, list of trials).

    make_case(i) (i = 0 for the warm-up, then 1, 2, ...) returns a dict with
    keys descriptors (device tensor of mt_subbatch records), num_subbatches,
    total, max_key_length, max_value_length (and anything that must stay
    alive while it runs).  trial(tree, case, config, stream) -> Mops/s runs
    one measurement (time_trial by default)."""
    if stream is None and trial is time_trial:
        import torch
        stream = torch.cuda.current_stream()
    trials = []
    t_start = time.time()

    # Untimed warm-up of every kernel flavour the search launches (module
    # loading and first-call set-up would otherwise land in the first trials);
    # one case serves them all.
    warm = make_case(0)
    for fm in forms:
        for ft in find_tiles:
            for wt in write_tiles:
                trial(tree, warm, dict(form=fm, find_tile=ft, write_tile=wt, bucketing=False, blocks_per_sm=0),
                      stream)
    del warm

    def run(config):
        mops = trial(tree, make_case(len(trials) + 1), config, stream)
        trials.append(dict(config, mops=round(mops, 2)))
        if log:
            log(trials[-1])
        return mops

    best, best_mops = None, -1.0
    for fm in forms:
        for ft in find_tiles:
            for wt in write_tiles:
                for bk in (bucketing if fm != "grouped" else (False,)):
                    cfg = dict(form=fm, find_tile=ft, write_tile=wt, bucketing=bk, blocks_per_sm=0)
                    m = run(cfg)
                    if m > best_mops:
                        best, best_mops = cfg, m
    for b in blocks_per_sm:
        cfg = dict(best, blocks_per_sm=b)
        m = run(cfg)
        if m > best_mops:
            best, best_mops = cfg, m
    return dict(best, mops=round(best_mops, 2), seconds=round(time.time() - t_start, 1)), trials
