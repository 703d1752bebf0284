"""Seeded synthetic workloads for the masstree benchmarks and parity tests.

Counterpart of the reference's evaluation/generate_workload.hpp, restated with
a counter-based generator so that any slice of a workload can be regenerated
independently (and identically) by tests and benchmarks:

  c1 (plain, small): keys of 1-8 uniform random slices, 2-slice values; finds
      are 50% hits sampled from the inserted keys and 50% fresh misses.
  c2 (mixed): keys of 2-16 slices = the first min(4, L-1) slices of one of 4096
      random 4-slice prefixes, random middle slices, and a last slice holding a
      Feistel-permuted unique id (reference feistel_permute,
      generate_workload.hpp:54-80); values of 1-8 slices, every slice the
      reference's key_hasher of the key (generate_workload.hpp:122-129).
      Batches mix 50% find / 30% insert (fresh ids) / 10% update / 10% erase,
      shuffled, with find/update/erase keys drawn Zipf(theta) over the preloaded
      ids by the reference's zipfian_int_distribution
      (generate_workload.hpp:82-120).
  c3 (scan): fixed 2-slice keys from uniform u64 (big-endian slices), 1-slice
      values, uniform random lower bounds.

The public benchmarks and datasets the reference can read (Memetracker, YCSB)
are not used; these seeded synthetic inputs have the configurations' shapes.
"""
import numpy as np

U64 = np.uint64
M64 = (1 << 64) - 1
REQ_INSERT, REQ_ERASE, REQ_FIND, REQ_UPDATE = 0, 1, 2, 3


def fmix64(x):
    """MurmurHash3 64-bit finalizer (wrapping uint64 arithmetic)."""
    x = np.asarray(x, dtype=U64)
    with np.errstate(over="ignore"):
        x = x ^ (x >> U64(33))
        x = x * U64(0xFF51AFD7ED558CCD)
        x = x ^ (x >> U64(33))
        x = x * U64(0xC4CEB9FE1A85EC53)
        x = x ^ (x >> U64(33))
    return x


def rnd64(seed, stream, idx):
    """Counter-based random u64 for (seed, stream, idx)."""
    idx = np.asarray(idx, dtype=U64)
    with np.errstate(over="ignore"):
        base = fmix64(U64((seed * 0x9E3779B97F4A7C15 + stream * 0xD1B54A32D192ED03) & M64))
        return fmix64(base + idx * U64(0x94D049BB133111EB))


def rnd32(seed, stream, idx):
    return (rnd64(seed, stream, idx) >> U64(32)).astype(np.uint32)


def uniform01(seed, stream, idx):
    """Uniform doubles in [0, 1)."""
    return (rnd64(seed, stream, idx) >> U64(11)).astype(np.float64) * (1.0 / (1 << 53))


def feistel_permute(x, n, seed=0):
    """Bijection of [0, n): 4-round Feistel network with cycle walking
    (the reference's feistel_permute, generate_workload.hpp:54-80)."""
    x = np.asarray(x, dtype=U64).copy()
    if n <= 1:
        return np.zeros_like(x)
    half = 0
    while (1 << (2 * half)) < n:
        half += 1
    mask = U64((1 << half) - 1)
    h = U64(half)
    out = np.empty_like(x)
    todo = np.arange(len(x))
    cur = x
    with np.errstate(over="ignore"):
        while len(todo):
            L, R = cur >> h, cur & mask
            for r in range(4):
                t = L
                L = R
                R = t ^ (fmix64(R + U64(seed + r)) & mask)
            cur = (L << h) | R
            ok = cur < U64(n)
            out[todo[ok]] = cur[ok]
            todo, cur = todo[~ok], cur[~ok]
    return out


def key_hasher(keys, lens):
    """The reference's key_hasher (generate_workload.hpp:122-129) with
    std::hash<uint32_t> the identity (libstdc++); returns the low 32 bits."""
    n, maxK = keys.shape
    h = np.zeros(n, dtype=U64)
    with np.errstate(over="ignore"):
        for s in range(maxK):
            live = lens > s
            k = keys[:, s].astype(U64)
            nh = h ^ (k + U64(0x9E3779B9) + (h << U64(6)) + (h >> U64(2)))
            h = np.where(live, nh, h)
    return h.astype(np.uint32)


_ZETA = {}


def zipf_sample(n_items, theta, u):
    """The reference's zipfian_int_distribution(0, n_items-1, theta) driven by
    uniform u in [0, 1] (generate_workload.hpp:82-120)."""
    key = (n_items, theta)
    if key not in _ZETA:
        zetan = float(np.sum(np.power(np.arange(1, n_items + 1, dtype=np.float64), -theta)))
        zeta2 = 1.0 + 0.5 ** theta
        _ZETA[key] = zetan, zeta2
    zetan, zeta2 = _ZETA[key]
    alpha = 1.0 / (1.0 - theta)
    eta = (1 - np.power(2.0 / n_items, 1 - theta)) / (1 - zeta2 / zetan)
    uz = u * zetan
    base = (n_items - 1) * np.power(eta * u - eta + 1, alpha)
    base = np.where(uz < 1.0, 0, np.where(uz < 1.0 + 0.5 ** theta, 1, base.astype(np.int64)))
    return np.clip(base, 0, n_items - 1).astype(np.int64)


# ---- C1 -------------------------------------------------------------------------

def c1_keys(n, seed=0xC1, first_id=0, maxK=8):
    """n distinct random keys of 1..maxK slices (ids first_id.. of stream `seed`)."""
    ids = np.arange(first_id, first_id + n, dtype=np.int64)
    lens = (1 + rnd32(seed, 0, ids) % np.uint32(maxK)).astype(np.uint32)
    keys = np.zeros((n, maxK), np.uint32)
    for s in range(maxK):
        col = rnd32(seed, 1 + s, ids)
        keys[:, s] = np.where(lens > s, col, 0)
    return keys, lens


def dedupe_rows(keys, lens):
    """Indices of the first occurrence of every distinct (key, length) row."""
    rows = np.concatenate([keys, lens[:, None]], axis=1)
    v = np.ascontiguousarray(rows).view(np.dtype((np.void, rows.dtype.itemsize * rows.shape[1])))
    _, first = np.unique(v.ravel(), return_index=True)
    return np.sort(first)


def c1(n_keys=1 << 20, n_finds=1 << 20, seed=0xC1, maxK=8, maxV=2):
    """Plain small workload: insert n_keys, then n_finds finds (50% hits)."""
    keys, lens = c1_keys(int(n_keys * 1.01) + 64, seed, 0, maxK)
    keep = dedupe_rows(keys, lens)[:n_keys]
    keys, lens = keys[keep], lens[keep]
    assert len(keys) == n_keys
    ids = np.arange(n_keys, dtype=np.int64)
    vals = np.stack([rnd32(seed + 1, s, ids) for s in range(maxV)], axis=1)
    vlens = np.full(n_keys, maxV, np.uint32)
    n_hit = n_finds // 2
    hit_idx = (rnd64(seed + 2, 0, np.arange(n_hit)) % U64(n_keys)).astype(np.int64)
    mk, ml = c1_keys(n_finds - n_hit + 64, seed + 3, 0, maxK)
    # Misses must be absent from the inserted set.
    allk = np.concatenate([keys, mk]), np.concatenate([lens, ml])
    firsts = dedupe_rows(*allk)
    fresh = firsts[firsts >= n_keys] - n_keys
    mk, ml = mk[fresh][: n_finds - n_hit], ml[fresh][: n_finds - n_hit]
    fkeys = np.concatenate([keys[hit_idx], mk])
    flens = np.concatenate([lens[hit_idx], ml])
    order = np.argsort(rnd64(seed + 4, 0, np.arange(n_finds)))
    return dict(keys=keys, lens=lens, vals=vals, vlens=vlens, find_keys=fkeys[order], find_lens=flens[order],
                find_hit=(np.concatenate([np.ones(n_hit, bool), np.zeros(len(mk), bool)]))[order],
                find_src=np.concatenate([hit_idx, -np.ones(len(mk), np.int64)])[order], maxK=maxK, maxV=maxV)


# ---- C2 -------------------------------------------------------------------------

class C2:
    """Mixed workload over 2..16-slice keys with 4096 shared 4-slice prefixes."""

    def __init__(self, n_preload=1 << 24, seed=0xC2, n_prefixes=4096, maxK=16, maxV=8, theta=0.99, id_space=1 << 32):
        self.n_preload, self.seed, self.maxK, self.maxV, self.theta = n_preload, seed, maxK, maxV, theta
        self.id_space = id_space
        pid = np.arange(n_prefixes * 4, dtype=np.int64)
        self.prefixes = rnd32(seed, 100, pid).reshape(n_prefixes, 4)
        self.n_prefixes = n_prefixes

    def keys(self, ids):
        """Keys and value payloads of key ids (ids < id_space are unique keys)."""
        ids = np.asarray(ids, dtype=np.int64)
        n = len(ids)
        maxK = self.maxK
        L = (2 + rnd32(self.seed, 1, ids) % np.uint32(maxK - 1)).astype(np.uint32)
        pfx = self.prefixes[(rnd32(self.seed, 2, ids) % np.uint32(self.n_prefixes)).astype(np.int64)]
        p = np.minimum(4, L - 1)
        uid = feistel_permute(ids.astype(U64), self.id_space, self.seed).astype(np.uint32)
        keys = np.zeros((n, maxK), np.uint32)
        for s in range(maxK):
            rand = rnd32(self.seed, 10 + s, ids)
            col = np.where(s < p, pfx[:, min(s, 3)], rand)
            col = np.where(s == L - 1, uid, col)
            keys[:, s] = np.where(s < L, col, 0)
        vl = (1 + rnd32(self.seed, 3, ids) % np.uint32(self.maxV)).astype(np.uint32)
        h = key_hasher(keys, L)
        vals = np.where(np.arange(self.maxV)[None, :] < vl[:, None], h[:, None], 0).astype(np.uint32)
        return keys, L, vals, vl

    def batch(self, b, n, mix=(0.5, 0.3, 0.1, 0.1)):
        """Mixed batch b of n requests (deterministic in (seed, b))."""
        nf = int(round(n * mix[0]))
        ni = int(round(n * mix[1]))
        nu = int(round(n * mix[2]))
        ne = n - nf - ni - nu
        types = np.concatenate([np.full(nf, REQ_FIND, np.uint8), np.full(ni, REQ_INSERT, np.uint8),
                                np.full(nu, REQ_UPDATE, np.uint8), np.full(ne, REQ_ERASE, np.uint8)])
        idx = np.arange(n, dtype=np.int64)
        u = uniform01(self.seed + 7, 1000 + b, idx)
        zipf_ids = zipf_sample(self.n_preload, self.theta, u)
        fresh_ids = self.n_preload + b * n + idx  # unique across batches
        ids = np.where(types == REQ_INSERT, fresh_ids, zipf_ids)
        order = np.argsort(rnd64(self.seed + 8, 1000 + b, idx), kind="stable")
        types, ids = types[order], ids[order]
        keys, lens, vals, vlens = self.keys(ids)
        upd = types == REQ_UPDATE
        with np.errstate(over="ignore"):
            newv = (vals.astype(U64) ^ (U64((b + 1) * 0x9E3779B1) & U64(0xFFFFFFFF))).astype(np.uint32)
        vals = np.where(upd[:, None] & (np.arange(self.maxV)[None, :] < vlens[:, None]), newv, vals)
        vals = np.where((types == REQ_FIND)[:, None], 0, vals).astype(np.uint32)
        vlens = np.where(types == REQ_FIND, 0, vlens).astype(np.uint32)
        return dict(types=types, ids=ids, keys=keys, lens=lens, vals=vals, vlens=vlens)


# ---- C3 -------------------------------------------------------------------------

def c3(n_keys, n_queries, seed=0xC3):
    """Fixed 8-byte keys (2 big-endian slices of a random u64), 1-slice values."""
    raw = rnd64(seed, 0, np.arange(int(n_keys * 1.001) + 64))
    raw = np.unique(raw)
    pick = np.argsort(rnd64(seed, 1, np.arange(len(raw))))[:n_keys]
    raw = raw[pick]
    keys = np.stack([(raw >> U64(32)).astype(np.uint32), (raw & U64(0xFFFFFFFF)).astype(np.uint32)], axis=1)
    vals = rnd32(seed, 2, np.arange(n_keys))[:, None]
    q = rnd64(seed, 3, np.arange(n_queries))
    lower = np.stack([(q >> U64(32)).astype(np.uint32), (q & U64(0xFFFFFFFF)).astype(np.uint32)], axis=1)
    return dict(keys=keys, lens=np.full(n_keys, 2, np.uint32), vals=vals, vlens=np.ones(n_keys, np.uint32),
                lower=lower, lower_lens=np.full(n_queries, 2, np.uint32))


# ---- C5 (serving) ---------------------------------------------------------------

def keys_threaded(c2, ids, threads=16):
    """c2.keys over chunks of ids in a thread pool (numpy releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    ids = np.asarray(ids, dtype=np.int64)
    n_chunks = max(1, min(threads, len(ids) // 65536))
    if n_chunks == 1:
        return c2.keys(ids)
    with ThreadPoolExecutor(n_chunks) as ex:
        parts = list(ex.map(c2.keys, np.array_split(ids, n_chunks)))
    return tuple(np.concatenate([p[i] for p in parts]) for i in range(4))


def serve_stream(c2, n_requests, rate_per_s=None, min_ops=1, max_ops=64, seed=0xC5, disjoint=False,
                 mix=(0.5, 0.3, 0.1, 0.1), first_fresh=None, op_seed=None, threads=16):
    """Open-loop request stream over a C2 tree of c2.n_preload keys.

    Request r holds a log-uniform number of ops in [min_ops, max_ops] of the
    C2 mix; arrivals are a Poisson process of rate_per_s requests per second
    (None: all at time 0).  disjoint=True draws find/update/erase keys without
    replacement from the preloaded ids (and half the finds from absent ids), so
    no two ops of the whole stream touch the same key and every op's result is
    independent of how requests interleave; otherwise they are Zipf(theta) as
    in c2 batches.  Inserts always use fresh ids (from first_fresh, default
    the middle of c2's id space, above the ids of its batches).  Sizes and
    arrivals follow `seed`, the ops `op_seed` (default: seed), so streams of
    equal shape and different content can be drawn.  Returns op arrays (types,
    ids, keys, lens, vals, vlens) and per-request first, nops, arrival_ns."""
    os_ = seed if op_seed is None else op_seed
    r = np.arange(n_requests, dtype=np.int64)
    u = uniform01(seed, 1, r)
    lo, hi = np.log(min_ops), np.log(max_ops + 1)
    nops = np.minimum(np.exp(lo + u * (hi - lo)).astype(np.int64), max_ops).astype(np.uint32)
    first = np.concatenate([[0], np.cumsum(nops[:-1], dtype=np.int64)]).astype(np.uint32)
    total = int(nops.sum(dtype=np.int64))
    idx = np.arange(total, dtype=np.int64)
    cum = np.cumsum(np.asarray(mix, np.float64))
    v = uniform01(os_, 2, idx)
    types = np.where(v < cum[0], REQ_FIND, np.where(v < cum[1], REQ_INSERT,
                                                    np.where(v < cum[2], REQ_UPDATE, REQ_ERASE))).astype(np.uint8)
    if first_fresh is None:
        first_fresh = c2.n_preload + c2.id_space // 2
    if first_fresh + total > c2.id_space:
        raise ValueError("fresh ids beyond the key id space")
    fresh = first_fresh + idx
    if disjoint:
        if total > c2.n_preload:
            raise ValueError("disjoint stream needs at least as many preloaded keys as ops")
        old = feistel_permute(idx.astype(U64), c2.n_preload, os_).astype(np.int64)
        miss = (types == REQ_FIND) & (rnd32(os_, 3, idx) & np.uint32(1)).astype(bool)
        ids = np.where((types == REQ_INSERT) | miss, fresh, old)
    else:
        ids = np.where(types == REQ_INSERT, fresh, zipf_sample(c2.n_preload, c2.theta, uniform01(os_, 4, idx)))
    keys, lens, vals, vlens = keys_threaded(c2, ids, threads)
    upd = types == REQ_UPDATE
    with np.errstate(over="ignore"):
        newv = (vals.astype(U64) ^ U64(0x5BD1E995)).astype(np.uint32)
    vals = np.where(upd[:, None] & (np.arange(c2.maxV)[None, :] < vlens[:, None]), newv, vals)
    vals = np.where((types == REQ_FIND)[:, None], 0, vals).astype(np.uint32)
    vlens = np.where(types == REQ_FIND, 0, vlens).astype(np.uint32)
    if rate_per_s is None:
        arrival = np.zeros(n_requests, np.uint64)
    else:
        gaps = -np.log1p(-uniform01(seed, 5, r)) / float(rate_per_s)
        arrival = (np.cumsum(gaps) * 1e9).astype(np.uint64)
    return dict(types=types, ids=ids, keys=keys, lens=lens.astype(np.uint32), vals=vals, vlens=vlens,
                first=first, nops=nops, arrival_ns=arrival)
