// Slab pool, per-tile slab cache and launch-granular reclamation.
//
// Replaces the reference's bitmap slab allocator (include/simple_slab_alloc.hpp:
// pool of 128-byte slabs addressed by u32 index, sized from a fraction of free
// device memory, :56-69) and its DEBRA reclaimer
// (include/simple_debra_reclaim.hpp: per-block epochs and limbo bags).
//
// Design (B200):
//   * The pool is split into S shards.  Each shard owns a contiguous slab range,
//     a bump counter, a LIFO free stack and a limbo list, each counter in its own
//     128-byte line so shards never contend.
//   * A tile refills T slabs at once (one atomic), one slab per lane, and hands
//     them out with a shuffle: one atomic per T allocations instead of one
//     bitmap fetch_or per allocation.
//   * retire() appends a slab to its home shard's limbo list.  Slabs retired
//     during launch k may still be read by other tiles of launch k; they are
//     moved to the free stacks by mt_reclaim_kernel, which runs stream-ordered
//     before the next launch on the tree.  No reader of launch k exists then, and
//     readers of launch k+1 cannot reach an unlinked slab.  That gives the same
//     guarantee as DEBRA's epochs with no per-round block barriers.
//   * Stack pops (atomicSub) and pushes (only in the reclaim kernel) never run
//     concurrently, so a plain counter stack is ABA-free.
//   * Every bounded failure (pool exhausted) records MT_ERR_OOM in the device
//     error word instead of spinning (the reference probes forever,
//     simple_slab_alloc.hpp:113-120).
#pragma once
#include "mt_tile.cuh"

namespace mtb {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kCtrStride = 32;  // ints: one 128-byte line per counter

enum mt_err_code : uint32_t {
  ERR_NONE = 0,
  ERR_OOM = 1,
  ERR_LOCK_TIMEOUT = 2,
  ERR_CORRUPT = 3,
  ERR_INVALID_ARG = 4,
  ERR_CUDA = 5,
  ERR_RETRY_LIMIT = 6,
  ERR_KEY_TOO_LONG = 7,
};

struct pool_view {
  uint32_t* slabs;        // slab i occupies words [32*i, 32*i+32)
  uint32_t* free_stack;   // [shards][shard_slabs]
  uint32_t* limbo;        // [shards][shard_slabs]
  int* ctr;               // per shard: top, bump, limbo count (each its own line)
  uint32_t* err;          // [0] first error code, [1] error count
  uint32_t num_slabs;
  uint32_t num_shards;
  uint32_t shard_slabs;
  uint32_t lock_spins;    // lock attempts before MT_ERR_LOCK_TIMEOUT (mt_set_lock_wait)

  MT_HD uint32_t* addr(uint32_t i) const { return slabs + (size_t)i * 32u; }
  MT_HD bool valid(uint32_t i) const { return i < num_slabs; }
  MT_HD int* top(uint32_t s) const { return ctr + (size_t)(3u * s + 0u) * kCtrStride; }
  MT_HD int* bump(uint32_t s) const { return ctr + (size_t)(3u * s + 1u) * kCtrStride; }
  MT_HD int* limbo_count(uint32_t s) const { return ctr + (size_t)(3u * s + 2u) * kCtrStride; }
};

// Where an error was detected: a source file number (high 16 bits) and line.
#define MT_AT(file) ((((uint32_t)(file)) << 16) | (uint32_t)__LINE__)
enum mt_src_file : uint32_t { SRC_TREE = 1, SRC_NODE = 2, SRC_SUFFIX = 3, SRC_POOL = 4, SRC_FIND = 5, SRC_CAPI = 6,
                              SRC_MERGE = 7, SRC_BULK = 8, SRC_SERVE = 9 };

// err[0] = first error code, err[1] = error count, err[2] = fatal flag,
// err[3] = where the first error was detected (MT_AT; 0 if not given).  A
// fatal error (lock timeout, corruption, retry limit) makes every tile of the
// launch stop taking new requests, so one failure cannot turn into a long
// series of bounded waits.
MT_DEV void record_error(const pool_view& p, uint32_t code, uint32_t site = 0u) {
  if (atomicCAS(p.err, 0u, code) == 0u) atomicExch(p.err + 3, site);
  atomicAdd(p.err + 1, 1u);
  if (code == ERR_LOCK_TIMEOUT || code == ERR_CORRUPT || code == ERR_RETRY_LIMIT) atomicExch(p.err + 2, 1u);
}
MT_DEV bool fatal_error(const pool_view& p) { return ld_relaxed_u32(p.err + 2) != 0u; }

// Per-tile slab cache: lane r holds one slab while r < count.
template <int T>
struct slab_cache {
  uint32_t slab = kInvalid;
  uint32_t count = 0;   // uniform over the tile
  uint32_t shard = 0;   // uniform: preferred shard

  MT_DEV void init(const pool_view& p, uint32_t tile_id) {
    slab = kInvalid;
    count = 0;
    shard = (tile_id * 0x9E3779B1u) % p.num_shards;
  }

  // Refill from one shard; returns number of slabs obtained (uniform).
  MT_DEV uint32_t refill_from(const tile<T>& t, const pool_view& p, uint32_t s) {
    int stack_begin = 0, n_stack = 0, bump_begin = 0, n_bump = 0;
    if (t.leader()) {
      int need = T;
      int* topp = p.top(s);
      if ((int)ld_relaxed_u32((const uint32_t*)topp) > 0) {
        int old = atomicSub(topp, need);
        if (old > 0) {
          int lo = old - need;
          if (lo < 0) lo = 0;
          stack_begin = lo;
          n_stack = old - lo;
          need -= n_stack;
        }
      }
      if (need > 0) {
        int* bp = p.bump(s);
        int cur = (int)ld_relaxed_u32((const uint32_t*)bp);
        if (cur < (int)p.shard_slabs) {
          int b = atomicAdd(bp, need);
          if (b < (int)p.shard_slabs) {
            bump_begin = b;
            n_bump = min(need, (int)p.shard_slabs - b);
          }
        }
      }
    }
    stack_begin = (int)t.shfl((uint32_t)stack_begin, 0);
    n_stack = (int)t.shfl((uint32_t)n_stack, 0);
    bump_begin = (int)t.shfl((uint32_t)bump_begin, 0);
    n_bump = (int)t.shfl((uint32_t)n_bump, 0);
    const int r = (int)t.rank;
    if (r < n_stack) {
      slab = ld_relaxed_u32(p.free_stack + (size_t)s * p.shard_slabs + stack_begin + r);
    } else if (r < n_stack + n_bump) {
      slab = s * p.shard_slabs + (uint32_t)(bump_begin + (r - n_stack));
    } else {
      slab = kInvalid;
    }
    return (uint32_t)(n_stack + n_bump);
  }

  // Returns a fresh slab index (uniform) or kInvalid after recording MT_ERR_OOM.
  MT_DEV uint32_t allocate(const tile<T>& t, const pool_view& p) {
    if (count == 0) {
      for (uint32_t k = 0; k < p.num_shards && count == 0; ++k) {
        const uint32_t s = (shard + k) % p.num_shards;
        count = refill_from(t, p, s);
        if (count) shard = s;
      }
      if (count == 0) {
        if (t.leader()) record_error(p, ERR_OOM, MT_AT(SRC_POOL));
        return kInvalid;
      }
    }
    --count;
    return t.shfl(slab, (int)count);
  }

  // Unused cached slabs go to limbo so the next reclaim returns them.
  MT_DEV void release(const tile<T>& t, const pool_view& p);
};

// Retire one slab (called by one lane).  Safe to free after the current launch.
MT_DEV void retire_slab(const pool_view& p, uint32_t slab) {
  if (!p.valid(slab)) { record_error(p, ERR_CORRUPT, MT_AT(SRC_POOL)); return; }
  const uint32_t s = slab / p.shard_slabs;
  const int pos = atomicAdd(p.limbo_count(s), 1);
  if (pos >= (int)p.shard_slabs) { record_error(p, ERR_CORRUPT, MT_AT(SRC_POOL)); return; }
  p.limbo[(size_t)s * p.shard_slabs + pos] = slab;
}

template <int T>
MT_DEV void slab_cache<T>::release(const tile<T>& t, const pool_view& p) {
  if (t.rank < count && slab != kInvalid) retire_slab(p, slab);
  count = 0;
  slab = kInvalid;
}

}  // namespace mtb
