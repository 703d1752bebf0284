"""Range-sharded masstree over the ranks of a process group (one GPU each).

The key space is cut by the first key slice into world_size contiguous ranges;
rank r holds the keys whose first slice s satisfies (s * world_size) >> 32 == r
in its own tree (the same partition the oracle's multi-threaded form uses, so
every shard holds one contiguous run of the global key order).  A mixed batch
submitted on any rank is filed by owner, exchanged with one all-to-all of
request records, served by each owner as one local mixed batch, and the results
come back with a second all-to-all into the caller's order.  A scan runs on the
shard owning its lower bound; a scan that reaches the end of a shard before
max_count results continues on the next shard from that shard's smallest key
(one more exchange round per shard crossed).

The reference is single-GPU (include/kernels.hpp:97-98); this is the sharded
form of the same API.  Requests of one mixed batch have no order among each
other, as in the reference, so serving each shard's part as its own batch is
one of the batch's allowed orders.  The exchanges are torch.distributed
all_to_all_single calls (NCCL over NVLink between GPUs; gloo on CPU in tests).
"""
import numpy as np


def shard_of_slices(first, world):
    """Owner rank of each first key slice (a numpy uint32 array, or a torch
    tensor of the slices' 32-bit words)."""
    if hasattr(first, "to"):  # torch tensor
        import torch
        return ((first.to(torch.int64) & 0xFFFFFFFF) * world) >> 32
    return ((np.asarray(first, dtype=np.uint64) * np.uint64(world)) >> np.uint64(32)).astype(np.int64)


class GpuShard:
    """The local part of a sharded index: a GpuMasstree driven with device
    tensors (mt_mixed_batch / mt_scan)."""

    def __init__(self, tree, stream=0):
        self.tree, self.stream = tree, stream

    def mixed(self, types, keys, klens, vals, vlens):
        import torch
        n = len(types)
        res = torch.zeros(n, dtype=torch.bool, device=keys.device)
        if n:
            self.tree.mixed_batch(types, keys, keys.shape[1], klens, vals, vals.shape[1], vlens, res, n,
                                  stream=self.stream)
            self.tree.sync(self.stream)
        return vals, vlens, res

    def scan(self, lower, lower_lens, max_count, maxV):
        import torch
        nq, maxK = lower.shape
        dev = lower.device
        z = lambda *s: torch.zeros(s, dtype=torch.uint32, device=dev)  # noqa: E731
        counts, vals, vlens, keys, klens = z(nq), z(nq, max_count, maxV), z(nq, max_count), \
            z(nq, max_count, maxK), z(nq, max_count)
        if nq:
            self.tree.scan(lower, lower_lens, maxK, max_count, nq, counts=counts, values=vals, max_value_length=maxV,
                           value_lengths=vlens, out_keys=keys, out_key_lengths=klens, stream=self.stream)
            self.tree.sync(self.stream)
        return counts, vals, vlens, keys, klens


class ShardedMasstree:
    """Mixed batches and scans over a range-sharded index.

    `local` serves this rank's shard (GpuShard in production); tensors passed
    in live on the process group's device (cuda for NCCL, cpu for gloo) and
    hold uint32 slices (any 4-byte dtype: they are exchanged as raw words).
    Every rank must call mixed_batch / scan together (they are collective),
    each with its own requests (any number, 0 included)."""

    def __init__(self, local, max_key_length, max_value_length, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.local = local
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.maxK, self.maxV = max_key_length, max_value_length

    # ---- exchange helpers -----------------------------------------------------
    def _exchange(self, rows, send_counts):
        """all-to-all of int32 rows filed by destination rank; returns (rows
        received, counts received)."""
        import torch
        sc = send_counts.to(torch.int64)
        rc = torch.empty_like(sc)
        self.dist.all_to_all_single(rc, sc, group=self.group)
        ins, outs = sc.tolist(), rc.tolist()
        recv = torch.empty((sum(outs), rows.shape[1]), dtype=rows.dtype, device=rows.device)
        self.dist.all_to_all_single(recv, rows.contiguous(), output_split_sizes=outs, input_split_sizes=ins,
                                    group=self.group)
        return recv, rc

    def _back(self, rows, recv_counts, send_counts):
        """The reverse all-to-all: results to the ranks that sent the requests."""
        import torch
        outs, ins = send_counts.tolist(), recv_counts.tolist()
        back = torch.empty((sum(outs), rows.shape[1]), dtype=rows.dtype, device=rows.device)
        self.dist.all_to_all_single(back, rows.contiguous(), output_split_sizes=outs, input_split_sizes=ins,
                                    group=self.group)
        return back

    def _file(self, dest):
        """Stable order of requests by destination, and the count per rank."""
        import torch
        order = torch.argsort(dest, stable=True)
        return order, torch.bincount(dest, minlength=self.world)

    def _owner(self, first_words, lens):
        import torch
        dest = shard_of_slices(first_words, self.world)
        return torch.where(lens > 0, dest, torch.zeros_like(dest))

    # ---- mixed batch ------------------------------------------------------------
    def mixed_batch(self, types, keys, klens, vals, vlens):
        """(values, value lengths, results) in the caller's order, as one
        mt_mixed_batch over the whole index would give them (uint32 values and
        lengths, bool results)."""
        import torch
        K, V = self.maxK, self.maxV
        i32 = torch.int32
        n = types.shape[0]
        keys, klens, vals, vlens = (x.contiguous().view(i32) for x in (keys, klens, vals, vlens))
        order, counts = self._file(self._owner(keys[:, 0], klens))
        rec = torch.cat([types.to(i32).view(n, 1), klens.view(n, 1), keys.view(n, K), vlens.view(n, 1),
                         vals.view(n, V)], dim=1)[order]
        got, rcounts = self._exchange(rec, counts)
        m = got.shape[0]
        o_vals, o_vlens, o_res = self.local.mixed(
            got[:, 0].to(torch.uint8).contiguous(), got[:, 2:2 + K].contiguous().view(torch.uint32),
            got[:, 1].contiguous().view(torch.uint32), got[:, 3 + K:3 + K + V].contiguous().view(torch.uint32),
            got[:, 2 + K].contiguous().view(torch.uint32))
        out = torch.cat([o_vlens.contiguous().view(i32).view(m, 1), o_res.to(i32).view(m, 1),
                         o_vals.contiguous().view(i32).view(m, V)], dim=1)
        back = self._back(out, rcounts, counts)
        rows = torch.empty_like(back)
        rows[order] = back
        return (rows[:, 2:2 + V].contiguous().view(torch.uint32), rows[:, 0].contiguous().view(torch.uint32),
                rows[:, 1] != 0)

    # ---- scan -------------------------------------------------------------------
    def scan(self, lower, lower_lens, max_count):
        """Ordered scans of up to max_count keys from each inclusive lower bound
        (no upper bound).  Returns counts, values, value lengths, keys and key
        lengths shaped as mt_scan's outputs (uint32)."""
        import torch
        K, V, W = self.maxK, self.maxV, self.world
        i32, i64 = torch.int32, torch.int64
        nq = lower.shape[0]
        dev = lower.device
        lower = lower.contiguous().view(i32).clone()
        lens = lower_lens.contiguous().view(i32).clone()
        counts = torch.zeros(nq, dtype=i64, device=dev)
        out = torch.zeros((nq, max_count, 2 + V + K), dtype=i32, device=dev)  # vlen, klen, value, key
        # Round 0 goes to the owner of the lower bound; each later round sends
        # the scans still short of max_count to the next shard, from its
        # smallest key.  Every rank takes part in all W rounds.
        shard = self._owner(lower[:, 0], lens)
        active = torch.ones(nq, dtype=torch.bool, device=dev)
        steps = torch.arange(max_count, device=dev)
        for _ in range(W):
            idx = torch.nonzero(active, as_tuple=False).view(-1)
            order, cnt = self._file(shard[idx])
            sel = idx[order]
            want = (max_count - counts[sel]).to(i32)
            rec = torch.cat([lens[sel].view(-1, 1), want.view(-1, 1), lower[sel]], dim=1)
            got, rcnt = self._exchange(rec, cnt)
            m = got.shape[0]
            c, v, vl, k, kl = self.local.scan(got[:, 2:].contiguous().view(torch.uint32),
                                              got[:, 0].contiguous().view(torch.uint32), max_count, V)
            c = torch.minimum(c.contiguous().view(i32).to(i64), got[:, 1].to(i64)).to(i32)
            per = torch.cat([vl.contiguous().view(i32).view(m, max_count, 1),
                             kl.contiguous().view(i32).view(m, max_count, 1),
                             v.contiguous().view(i32).view(m, max_count, V),
                             k.contiguous().view(i32).view(m, max_count, K)], dim=2)
            back = self._back(torch.cat([c.view(m, 1), per.reshape(m, max_count * (2 + V + K))], dim=1), rcnt, cnt)
            b_cnt = back[:, 0].to(i64)
            b_rows = back[:, 1:].view(-1, max_count, 2 + V + K)
            # Each query's new results go after its earlier ones.
            valid = steps.view(1, -1) < b_cnt.view(-1, 1)
            qq = sel.view(-1, 1).expand(-1, max_count)
            pos = counts[sel].view(-1, 1) + steps.view(1, -1)
            out[qq[valid], pos[valid]] = b_rows[valid]
            counts[sel] += b_cnt
            # Continue on the next shard from its smallest key.
            nxt = shard + 1
            active = active & (counts < max_count) & (nxt < W)
            shard = torch.where(active, nxt, shard)
            low = ((shard.to(i64) << 32) + (W - 1)) // W  # smallest first slice of the shard
            lower = torch.where(active.view(-1, 1), torch.zeros_like(lower), lower)
            low_word = ((low + (1 << 31)) % (1 << 32) - (1 << 31)).to(i32)  # the slice's 32-bit word
            lower[:, 0] = torch.where(active, low_word, lower[:, 0])
            lens = torch.where(active, torch.ones_like(lens), lens)
        u32 = torch.uint32
        return (counts.to(i32).view(u32), out[:, :, 2:2 + V].contiguous().view(u32),
                out[:, :, 0].contiguous().view(u32), out[:, :, 2 + V:].contiguous().view(u32),
                out[:, :, 1].contiguous().view(u32))
