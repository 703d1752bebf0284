// Device API of the B200 masstree: tile-cooperative find / insert / update /
// erase / scan over a trie of B-link trees (one B-link tree per 4-byte key
// slice).  These are the counterparts of the reference's
// gpu_masstree::cooperative_{find,insert,update,erase,scan}
// (include/gpu_masstree.hpp:194-248, 397-627, 629-749, 751-971, 250-395) and
// keep their observable semantics:
//   * find returns the FULL value length (0 = miss) and writes at most maxV
//     value slices;
//   * insert never overwrites unless update_if_exists; a key already present
//     makes it return false;
//   * update fails on a miss; erase returns whether the key was present;
//   * scan visits keys in lexicographic u32-slice order (a key that is a prefix
//     of another sorts first), both bounds inclusive.
//
// Concurrency: readers are lock-free.  The reference assumes one coalesced
// 128-byte load observes a concurrent 128-byte store atomically
// (README.md:168-172); on B200 that assumption fails about once in 10^5
// contended reads, so every lock-free node load here is checked against the
// node's checksum and reloaded on a mismatch (mt_node.cuh).  Writers lock a
// node through its meta word, publish the new node image with release stores
// and release the lock with a separate release atomic.  Inserts
// split full nodes top-down on the way to the border node (the proactive
// B-link split of Awad et al., "Engineering a High-Performance GPU B-Tree",
// PPoPP 2019, which the reference also uses, include/gpu_masstree.hpp:1020-1148).
// Erase removes entries without merging nodes (the reference's merge_level 0);
// on request it logs sparse border nodes and emptied trie layers, which a pass
// after the call merges or removes (mt_merge.cu).  Results are the same either
// way; only the space differs.  Every spin and every retry
// loop is bounded and records an error code instead of hanging.
#pragma once
#include "mt_suffix.cuh"

namespace mtb {

constexpr uint32_t kMaxHops = 1u << 16;     // node visits per operation
constexpr uint32_t kLockSpins = 1u << 20;   // default lock attempts (about 1 s) before MT_ERR_LOCK_TIMEOUT
constexpr uint32_t kMaxRestarts = 1u << 14;
#ifndef MT_LOCK_POLLS
#define MT_LOCK_POLLS 0
#endif
constexpr uint32_t kLockPolls = MT_LOCK_POLLS;  // lock retries without a sleep before the backoff starts

#ifndef MT_CONC_LOAD
#define MT_CONC_LOAD ::mtb::ld_order::RELAXED
#endif
// Order of lock-free node loads in operations that run beside writers.
// Relaxed gpu-scope loads are served by L2, the point of coherence, so a
// pointer read from a published node leads to the already-published target;
// the node checksum rejects any image that is torn or not yet written.
constexpr ld_order kConc = MT_CONC_LOAD;
// Suffix chains are immutable after publication; they are read after the
// owning entry was read with kConc, from L2.
constexpr ld_order kConcSuffix = ld_order::RELAXED;

enum op_result : int { RES_ERR = -1, RES_FAIL = 0, RES_OK = 1 };

struct tree_view {
  pool_view pool;
  uint32_t root;  // root slab of trie layer 0 (never moves)
  // Merge log of the current call, null unless the call merges sparse nodes
  // after its erases: [0] records, [1] unused, then one (layer root, slice)
  // pair per border node that an erase left with kMergeAt entries or none.
  uint32_t* merge_log;
  uint32_t merge_cap;
  // Layer log of the current call, null unless the call removes the trie
  // layers that its erases empty: [0] records, [1] unused, then records of
  // kLayerRecWords words, {layer, key slices 0 .. layer-1}, one per erase
  // that left the only node of a layer (layer 1 or deeper) without entries,
  // or (when the call merges too) the layer's rightmost border node.
  uint32_t* layer_log;
  uint32_t layer_cap;
};

// Words per layer-log record; layers deeper than kLayerRecWords-1 are not
// logged (and so never removed; the space stays in use, results are the same).
constexpr uint32_t kLayerRecWords = 16;

// A border node with this many entries or fewer after an erase is a merge
// candidate (of kMaxEntries = 13), and so is an interior node that a merge
// of its children leaves with this many.
constexpr uint32_t kMergeAt = 4;

// ---- locking -----------------------------------------------------------------

template <int T>
MT_DEV void unlock_node(const tile<T>& t, const pool_view& p, uint32_t idx) {
  t.sync();
  if (t.leader()) atom_and_release(p.addr(idx) + WORD_META, ~META_LOCK);
  t.sync();
}

// The first attempt goes straight to the atomic (an uncontended lock costs one
// round trip); after a failure it is test-and-test-and-set: waiters poll the
// meta word with plain loads and only try the atomic when it reads unlocked,
// with jittered exponential backoff (64 ns .. 1 us), so a hot node's holder is
// not slowed by a storm of atomics on its line.
template <int T>
MT_DEV bool lock_load(const tile<T>& t, const pool_view& p, uint32_t idx, node<T>& nd) {
  uint32_t* mw = p.addr(idx) + WORD_META;
  uint32_t backoff = 64u;
  uint32_t jitter = (idx * 0x9E3779B1u) ^ (uint32_t)clock();
  for (uint32_t it = 0; it < p.lock_spins; ++it) {
    uint32_t old = META_LOCK;
    if (t.leader()) {
      if (it == 0u || !(ld_relaxed_u32(mw) & META_LOCK)) old = atom_or_acquire(mw, META_LOCK);
    }
    old = t.shfl(old, 0);
    if (!(old & META_LOCK)) {
      t.sync();
      // No writer can publish this node while we hold its lock; a checksum
      // mismatch here would be a bug, reported as corruption.
      return nd.template load_verified<ld_order::ACQUIRE>(t, p, idx) || (unlock_node(t, p, idx), false);
    }
    if ((it & 255u) == 255u && t.shfl((uint32_t)(t.leader() && fatal_error(p)), 0)) return false;
    // The first retries poll (a holder usually releases within a few hundred
    // nanoseconds); later ones sleep with jittered exponential backoff.
    if (it + 1u > kLockPolls) {
      jitter = jitter * 1664525u + 1013904223u;
      __nanosleep(backoff + ((jitter >> 16) & (backoff - 1u)));
      if (backoff < 512u) backoff <<= 1;
    }
  }
  if (t.leader()) record_error(p, ERR_LOCK_TIMEOUT, MT_AT(SRC_TREE));
  return false;
}

// Publish the node image; the stored meta keeps LOCK set.
template <int T>
MT_DEV void publish_locked(const tile<T>& t, const pool_view& p, node<T>& nd) {
  nd.meta = (nd.meta | META_LOCK) + META_VERSION_ONE;
  nd.encode_header(t);
  nd.seal(t);
  nd.template store<st_order::RELEASE>(t, p);
}

// Publish the node image, then release its lock.  The release is a separate
// atomic after the image store (release-ordered): a line store is not seen
// atomically on B200, and a next holder must not take the lock before every
// word of this image has landed.  (Clearing LOCK in the image store itself,
// which saves the atomic, produced corrupted nodes under contention.)
template <int T>
MT_DEV void publish_unlock(const tile<T>& t, const pool_view& p, node<T>& nd) {
  publish_locked(t, p, nd);
  unlock_node(t, p, nd.idx);
  nd.meta &= ~META_LOCK;
}

// Write a node that no other tile can reach yet.
template <int T>
MT_DEV void publish_new(const tile<T>& t, const pool_view& p, node<T>& nd) {
  nd.encode_header(t);
  nd.seal(t);
  nd.template store<st_order::RELEASE>(t, p);
}

// Fresh layer root (an empty border node covering every slice).
template <int T>
MT_DEV void make_layer_root(const tile<T>& t, node<T>& nd, uint32_t idx) {
  nd.clear_words();
  nd.idx = idx;
  nd.meta = META_BORDER | META_ROOT;
  nd.ks = 0u;
  nd.high = 0xFFFFFFFFu;
  nd.sib = kInvalid;
}

// ---- descents ------------------------------------------------------------------

// Lock-free descent of one layer to the border node covering `slice`.
template <int T, ld_order O>
MT_DEV bool descend(const tile<T>& t, const pool_view& p, uint32_t root, uint32_t slice,
                    node<T>& nd, uint32_t& hops, uint32_t hop_limit = kMaxHops) {
  uint32_t idx = root;
  while (true) {
    if (!p.valid(idx) || ++hops > hop_limit) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE));
      return false;
    }
    if (!nd.template load_verified<O>(t, p, idx)) return false;
    if (nd.must_move_right(slice)) { idx = nd.sib; continue; }
    if (nd.is_border()) return true;
    const int c = nd.child_pos(t, slice);
    if (c < 0) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE));
      return false;
    }
    idx = nd.val_at(t, (uint32_t)c);
  }
}

// Lock the border node covering `slice`, starting from an unlocked image nd
// obtained by a lock-free descent.  Moves right and re-descends as needed.
template <int T>
MT_DEV bool lock_border(const tile<T>& t, const pool_view& p, uint32_t slice, node<T>& nd, uint32_t& hops) {
  uint32_t idx = nd.idx;
  while (true) {
    if (!p.valid(idx) || ++hops > kMaxHops) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE));
      return false;
    }
    if (!lock_load(t, p, idx, nd)) return false;
    if (nd.must_move_right(slice)) {
      unlock_node(t, p, idx);
      idx = nd.sib;
      continue;
    }
    if (!nd.is_border()) {  // a layer root split after the lock-free descent
      unlock_node(t, p, idx);
      if (!descend<T, kConc>(t, p, idx, slice, nd, hops)) return false;
      idx = nd.idx;
      continue;
    }
    return true;
  }
}

// Split position of a full node: never between the two entries of one slice.
template <int T>
MT_DEV uint32_t split_pos(const tile<T>& t, const node<T>& nd) {
  uint32_t p = kMaxEntries / 2;
  if (nd.is_border() && nd.key_at(t, p - 1) == nd.key_at(t, p)) ++p;
  return p;
}

// Split the full node nd, locked by the caller (with its parent `parent` when
// nd is not a layer root).  Returns 0 with nd = the half covering `slice`
// (locked iff it is a border node) and parent updated; 1 when the parent
// changed and the layer must be descended again; -1 on error.  Nothing else is
// left locked.  (Kept inline: ptxas 12.9 crashes on an out-of-line version.)
template <int T>
MT_DEV int split_full(const tile<T>& t, const pool_view& p, slab_cache<T>& cache, uint32_t slice,
                                       node<T>& nd, uint32_t& parent, uint32_t& restarts) {
  const uint32_t idx = nd.idx;
  const uint32_t sp = split_pos(t, nd);
  const uint32_t left_high = nd.key_at(t, sp - 1);
  const bool go_right = slice > left_high;
  const bool border = nd.is_border();
  node<T> rn;
  if (nd.is_root()) {
    // The layer root keeps its slab: its entries move to two new children.
    const uint32_t L = cache.allocate(t, p);
    const uint32_t R = (L != kInvalid) ? cache.allocate(t, p) : kInvalid;
    if (R == kInvalid) {
      if (L != kInvalid && t.leader()) retire_slab(p, L);
      unlock_node(t, p, idx);
      return -1;
    }
    node<T> ln;
    rn.take_upper_from(t, nd, sp);
    rn.idx = R;
    rn.meta = (border ? META_BORDER : 0u) | (nd.count() - sp);
    rn.ks = border ? (nd.ks >> (2u * sp)) : 0u;
    rn.high = nd.high;
    rn.sib = kInvalid;
#pragma unroll
    for (int k = 0; k < node<T>::W; ++k) ln.w[k] = nd.w[k];
    ln.truncate(t, sp);
    ln.idx = L;
    ln.meta = (border ? META_BORDER : 0u) | META_SIB | sp;
    ln.ks = border ? (nd.ks & ((1u << (2u * sp)) - 1u)) : 0u;
    ln.high = left_high;
    ln.sib = R;
    // The child we continue into stays locked if it is a border node.
    if (go_right && border) rn.meta |= META_LOCK;
    if (!go_right && border) ln.meta |= META_LOCK;
    publish_new(t, p, rn);
    publish_new(t, p, ln);
    const uint32_t old_high = nd.high;
    nd.clear_words();
    nd.set_word(t, 0, left_high);
    nd.set_word(t, 1, L);
    nd.set_word(t, 2, old_high);
    nd.set_word(t, 3, R);
    nd.meta = (nd.meta & ~(META_COUNT | META_BORDER)) | 2u;
    nd.ks = 0u;
    publish_unlock(t, p, nd);
    parent = idx;
    if (go_right) {
      nd = rn;
    } else {
      nd = ln;
    }
  } else {
    if (parent == kInvalid || ++restarts > kMaxRestarts) {
      unlock_node(t, p, idx);
      if (restarts > kMaxRestarts) { if (t.leader()) record_error(p, ERR_RETRY_LIMIT, MT_AT(SRC_TREE)); return -1; }
      return 1;
    }
    node<T> pn;
    if (!lock_load(t, p, parent, pn)) { unlock_node(t, p, idx); return -1; }
    const int j = pn.is_border() ? -1 : pn.child_slot_of(t, idx);
    if (pn.full() || j < 0) {
      // The parent changed under us: start the layer again.
      unlock_node(t, p, parent);
      unlock_node(t, p, idx);
      if (++restarts > kMaxRestarts) { if (t.leader()) record_error(p, ERR_RETRY_LIMIT, MT_AT(SRC_TREE)); return -1; }
      return 1;
    }
    const uint32_t R = cache.allocate(t, p);
    if (R == kInvalid) {
      unlock_node(t, p, parent);
      unlock_node(t, p, idx);
      return -1;
    }
    rn.take_upper_from(t, nd, sp);
    rn.idx = R;
    rn.meta = (border ? META_BORDER : 0u) | (nd.meta & META_SIB) | (nd.count() - sp);
    rn.ks = border ? (nd.ks >> (2u * sp)) : 0u;
    rn.high = nd.high;
    rn.sib = nd.sib;
    if (go_right && border) rn.meta |= META_LOCK;
    nd.truncate(t, sp);
    nd.meta = (nd.meta & ~META_COUNT) | META_SIB | sp;
    nd.ks = border ? (nd.ks & ((1u << (2u * sp)) - 1u)) : 0u;
    nd.high = left_high;
    nd.sib = R;
    // Parent: (left_high -> idx) inserted at j; old entry j (-> idx) now -> R.
    pn.insert_at(t, (uint32_t)j, left_high, idx, 0u);
    pn.set_entry(t, (uint32_t)j + 1u, R, 0u);
    // Write order: right, left, parent.
    publish_new(t, p, rn);
    publish_locked(t, p, nd);
    publish_unlock(t, p, pn);
    if (go_right) {
      unlock_node(t, p, idx);
      nd = rn;
    }
    parent = pn.idx;  // both halves hang under pn
  }
  return 0;
}

// Descent of one layer for an insert, splitting full nodes on the way.
// Returns 0 with nd = the LOCKED, non-full border node covering `slice`;
// 1 when the border node already holds a LINK for (slice, continues) (link set,
// nothing locked); -1 on error.
template <int T>
MT_DEV int descend_split(const tile<T>& t, const pool_view& p, slab_cache<T>& cache, uint32_t root,
                         uint32_t slice, bool more, node<T>& nd, uint32_t& link, uint32_t& hops) {
  uint32_t parent = kInvalid;
  uint32_t idx = root;
  uint32_t restarts = 0;
  while (true) {
    if (!p.valid(idx) || ++hops > kMaxHops) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE));
      return -1;
    }
    if (!nd.template load_verified<kConc>(t, p, idx)) return -1;
    if (nd.must_move_right(slice)) { idx = nd.sib; continue; }
    if (nd.is_border() && more) {
      const int e = nd.match(t, slice, true);
      if (e >= 0 && ks_get(nd.ks, (uint32_t)e) == KS_LINK) { link = nd.val_at(t, (uint32_t)e); return 1; }
    }
    if (!nd.is_border() && !nd.full()) {
      const int c = nd.child_pos(t, slice);
      if (c < 0) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return -1; }
      parent = idx;
      idx = nd.val_at(t, (uint32_t)c);
      continue;
    }
    // Border node or full interior node: lock it.
    if (!lock_load(t, p, idx, nd)) return -1;
    if (nd.must_move_right(slice)) { unlock_node(t, p, idx); idx = nd.sib; continue; }
    if (!nd.full()) {
      if (nd.is_border()) return 0;
      unlock_node(t, p, idx);
      const int c = nd.child_pos(t, slice);
      if (c < 0) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return -1; }
      parent = idx;
      idx = nd.val_at(t, (uint32_t)c);
      continue;
    }
    // nd is full and locked: split it.
    const int sr = split_full(t, p, cache, slice, nd, parent, restarts);
    if (sr < 0) return -1;
    if (sr == 1) {
      // Start the layer again.  The node-visit bound (which catches cycles)
      // applies per attempt; attempts are bounded by kMaxRestarts.  Inserts
      // into a young tree, where every tile meets the same splitting nodes,
      // restart thousands of times.
      idx = root;
      parent = kInvalid;
      hops = 0;
      continue;
    }
    // nd is now the non-full half covering slice; locked iff border.
    if (nd.is_border()) {
      nd.meta |= META_LOCK;
      return 0;
    }
    if (nd.locked()) unlock_node(t, p, nd.idx);
    const int c = nd.child_pos(t, slice);
    if (c < 0) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return -1; }
    parent = nd.idx;
    idx = nd.val_at(t, (uint32_t)c);
  }
}

// ---- find ------------------------------------------------------------------------

template <int T, bool CONCURRENT>
MT_DEV uint32_t coop_find(const tile<T>& t, const tree_view& tv, const uint32_t* key, uint32_t klen,
                          uint32_t* out, uint32_t maxV) {
  constexpr ld_order O = CONCURRENT ? kConc : ld_order::NC;
  constexpr ld_order OS = CONCURRENT ? kConcSuffix : ld_order::NC;
  const pool_view& p = tv.pool;
  uint32_t root = tv.root, hops = 0;
  node<T> nd;
  for (uint32_t layer = 0; layer < klen; ++layer) {
    const uint32_t slice = key[layer];
    const bool more = layer + 1u < klen;
    if (!descend<T, O>(t, p, root, slice, nd, hops)) return 0u;
    const int e = nd.match(t, slice, more);
    if (e < 0) return 0u;
    const uint32_t st = ks_get(nd.ks, (uint32_t)e);
    const uint32_t v = nd.val_at(t, (uint32_t)e);
    if (st == KS_LINK) { root = v; continue; }
    if (st == KS_VALUE) {
      if (maxV > 0u && out != nullptr && t.leader()) out[0] = v;
      return 1u;
    }
    if (!p.valid(v)) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return 0u; }
    suffix_head<T> h;
    h.template load<OS>(t, p, v);
    if (st == KS_SUFFIX) {
      const uint32_t lk = klen - layer - 1u;
      if (h.klen != lk) return 0u;
      if (suffix_compare<T, OS>(t, p, h, key + layer + 1u, lk).sign != 0) return 0u;
    }
    return suffix_get_value<T, OS>(t, p, h, out, maxV);
  }
  return 0u;
}

// ---- helpers shared by insert and update -----------------------------------------

// New representation of a value: inline for length 1, else a LONGVAL chain.
template <int T>
MT_DEV bool make_value(const tile<T>& t, const pool_view& p, slab_cache<T>& cache,
                       const uint32_t* val, uint32_t vlen, uint32_t& nv, uint32_t& ns) {
  if (vlen == 1u) {
    nv = val[0];
    ns = KS_VALUE;
    return true;
  }
  slice_src k, v;
  v.ptr = val;
  v.len = vlen;
  nv = suffix_create<T, kConcSuffix>(t, p, cache, k, v);
  ns = KS_LONGVAL;
  return nv != kInvalid;
}

// Replace the value of entry e (VALUE/LONGVAL) of the locked border node.
template <int T>
MT_DEV int replace_value(const tile<T>& t, const pool_view& p, slab_cache<T>& cache, node<T>& nd,
                         uint32_t e, uint32_t old_state, uint32_t old_val, const uint32_t* val, uint32_t vlen) {
  uint32_t nv, ns;
  if (!make_value(t, p, cache, val, vlen, nv, ns)) {
    unlock_node(t, p, nd.idx);
    return RES_ERR;
  }
  nd.set_entry(t, e, nv, ns);
  publish_unlock(t, p, nd);
  if (old_state == KS_LONGVAL) suffix_retire<T, kConcSuffix>(t, p, old_val);
  return RES_OK;
}

// Replace a SUFFIX entry whose key rest equals K with a chain holding K + val.
template <int T>
MT_DEV int replace_suffix(const tile<T>& t, const pool_view& p, slab_cache<T>& cache, node<T>& nd,
                          uint32_t e, uint32_t old_chain, const uint32_t* K, uint32_t lk,
                          const uint32_t* val, uint32_t vlen) {
  slice_src ks, vs;
  ks.ptr = K;
  ks.len = lk;
  vs.ptr = val;
  vs.len = vlen;
  const uint32_t nv = suffix_create<T, kConcSuffix>(t, p, cache, ks, vs);
  if (nv == kInvalid) { unlock_node(t, p, nd.idx); return RES_ERR; }
  nd.set_entry(t, e, nv, KS_SUFFIX);
  publish_unlock(t, p, nd);
  suffix_retire<T, kConcSuffix>(t, p, old_chain);
  return RES_OK;
}

// Entry payload for a key tail: (slice at position m of K, state, value).
// K[0..lk) is the key rest after the border slice; `m` indexes it.
template <int T>
MT_DEV bool make_tail_entry(const tile<T>& t, const pool_view& p, slab_cache<T>& cache,
                            const slice_src& K, uint32_t lk, uint32_t m, const slice_src& V,
                            uint32_t& slice, uint32_t& state, uint32_t& value) {
  const bool more = m + 1u < lk;
  if (K.ptr) slice = K.ptr[m];
  else slice = chain_slice<kConcSuffix>(p, K.chain, K.offset + m);
  if (more) {
    slice_src rest = K;
    if (rest.ptr) rest.ptr += m + 1u;
    else rest.offset += m + 1u;
    rest.len = lk - m - 1u;
    value = suffix_create<T, kConcSuffix>(t, p, cache, rest, V);
    state = KS_SUFFIX;
    return value != kInvalid;
  }
  if (V.len == 1u) {
    value = V.ptr ? V.ptr[0] : chain_slice<kConcSuffix>(p, V.chain, V.offset);
    state = KS_VALUE;
    return true;
  }
  slice_src none;
  value = suffix_create<T, kConcSuffix>(t, p, cache, none, V);
  state = KS_LONGVAL;
  return value != kInvalid;
}

// Two keys share a SUFFIX entry's slice but differ later: replace the entry by a
// LINK to a chain of single-entry layers for the common slices, ending in a layer
// with one entry per key (the reference's singleton/doubleton conversion,
// include/gpu_masstree.hpp:533-577).
template <int T>
MT_DEV int split_suffix(const tile<T>& t, const pool_view& p, slab_cache<T>& cache, node<T>& nd,
                        uint32_t e, const suffix_head<T>& h, uint32_t first_diff,
                        const uint32_t* K, uint32_t lk, const uint32_t* val, uint32_t vlen) {
  const uint32_t ls = h.klen;
  const uint32_t m = min(first_diff, min(ls, lk) - 1u);
  // Old key tail and value live in the old chain.
  slice_src oldK, oldV, newK, newV;
  oldK.chain = h.idx; oldK.offset = 0; oldK.len = ls;
  oldV.chain = h.idx; oldV.offset = ls; oldV.len = h.vlen;
  newK.ptr = K; newK.len = lk;
  newV.ptr = val; newV.len = vlen;
  uint32_t so, sto, vo, sn, stn, vn;
  if (!make_tail_entry(t, p, cache, oldK, ls, m, oldV, so, sto, vo)) { unlock_node(t, p, nd.idx); return RES_ERR; }
  if (!make_tail_entry(t, p, cache, newK, lk, m, newV, sn, stn, vn)) { unlock_node(t, p, nd.idx); return RES_ERR; }
  // Doubleton layer root.
  const uint32_t dslab = cache.allocate(t, p);
  if (dslab == kInvalid) { unlock_node(t, p, nd.idx); return RES_ERR; }
  node<T> ln;
  make_layer_root(t, ln, dslab);
  if (pos_less(so, ks_more(sto), sn, ks_more(stn))) {
    ln.insert_at(t, 0, so, vo, sto);
    ln.insert_at(t, 1, sn, vn, stn);
  } else {
    ln.insert_at(t, 0, sn, vn, stn);
    ln.insert_at(t, 1, so, vo, sto);
  }
  publish_new(t, p, ln);
  // Singleton layers for the common slices K[m-1] .. K[0], built bottom-up.
  uint32_t below = dslab;
  for (int i = (int)m - 1; i >= 0; --i) {
    const uint32_t s = cache.allocate(t, p);
    if (s == kInvalid) { unlock_node(t, p, nd.idx); return RES_ERR; }
    make_layer_root(t, ln, s);
    ln.insert_at(t, 0, K[i], below, KS_LINK);
    publish_new(t, p, ln);
    below = s;
  }
  nd.set_entry(t, e, below, KS_LINK);
  publish_unlock(t, p, nd);
  suffix_retire<T, kConcSuffix>(t, p, h.idx);
  return RES_OK;
}

// ---- insert ------------------------------------------------------------------------

template <int T, bool UPSERT>
MT_DEV int coop_insert(const tile<T>& t, const tree_view& tv, slab_cache<T>& cache, const uint32_t* key,
                       uint32_t klen, const uint32_t* val, uint32_t vlen) {
  const pool_view& p = tv.pool;
  if (klen == 0u || vlen > kMaxLen16 || klen > kMaxLen16) {
    if (t.leader()) record_error(p, ERR_INVALID_ARG, MT_AT(SRC_TREE));
    return RES_ERR;
  }
  uint32_t root = tv.root, hops = 0;
  node<T> nd;
  for (uint32_t layer = 0; layer < klen;) {
    const uint32_t slice = key[layer];
    const bool more = layer + 1u < klen;
    uint32_t link = kInvalid;
    const int r = descend_split(t, p, cache, root, slice, more, nd, link, hops);
    if (r < 0) return RES_ERR;
    if (r == 1) { root = link; ++layer; continue; }
    const int e = nd.match(t, slice, more);
    if (e >= 0) {
      const uint32_t st = ks_get(nd.ks, (uint32_t)e);
      const uint32_t v = nd.val_at(t, (uint32_t)e);
      if (st == KS_LINK) { unlock_node(t, p, nd.idx); root = v; ++layer; continue; }
      if (st == KS_VALUE || st == KS_LONGVAL) {
        if (!UPSERT) { unlock_node(t, p, nd.idx); return RES_FAIL; }
        return replace_value(t, p, cache, nd, (uint32_t)e, st, v, val, vlen);
      }
      // SUFFIX entry: same key, or a different key sharing this slice.
      if (!p.valid(v)) { unlock_node(t, p, nd.idx); if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return RES_ERR; }
      suffix_head<T> h;
      h.template load<kConcSuffix>(t, p, v);
      const uint32_t lk = klen - layer - 1u;
      const cmp_result c = suffix_compare<T, kConcSuffix>(t, p, h, key + layer + 1u, lk);
      if (c.sign == 0) {
        if (!UPSERT) { unlock_node(t, p, nd.idx); return RES_FAIL; }
        return replace_suffix(t, p, cache, nd, (uint32_t)e, v, key + layer + 1u, lk, val, vlen);
      }
      return split_suffix(t, p, cache, nd, (uint32_t)e, h, c.first_diff, key + layer + 1u, lk, val, vlen);
    }
    // Absent: add one entry.
    uint32_t nv, ns;
    if (more) {
      slice_src ks, vs;
      ks.ptr = key + layer + 1u;
      ks.len = klen - layer - 1u;
      vs.ptr = val;
      vs.len = vlen;
      nv = suffix_create<T, kConcSuffix>(t, p, cache, ks, vs);
      ns = KS_SUFFIX;
      if (nv == kInvalid) { unlock_node(t, p, nd.idx); return RES_ERR; }
    } else if (!make_value(t, p, cache, val, vlen, nv, ns)) {
      unlock_node(t, p, nd.idx);
      return RES_ERR;
    }
    nd.insert_at(t, nd.lower_pos(t, slice, more), slice, nv, ns);
    publish_unlock(t, p, nd);
    return RES_OK;
  }
  return RES_ERR;
}

// ---- lock-free presence check ------------------------------------------------------

// Whether the key (its slice at `layer` is the border slice) is present in a
// verified border image nd: returns 1 and the entry's value in *v if present,
// 0 if absent.  A consistent image read without the lock is a valid
// linearisation point for a miss, so update/erase/insert fail without locking.
template <int T>
MT_DEV int present_in_image(const tile<T>& t, const pool_view& p, const node<T>& nd, const uint32_t* key,
                            uint32_t klen, uint32_t layer, uint32_t* v) {
  const uint32_t slice = key[layer];
  const bool more = layer + 1u < klen;
  const int e = nd.match(t, slice, more);
  if (e < 0) return 0;
  const uint32_t st = ks_get(nd.ks, (uint32_t)e);
  *v = nd.val_at(t, (uint32_t)e);
  if (st != KS_SUFFIX) return 1;
  if (!p.valid(*v)) return 1;  // let the locked path report it
  suffix_head<T> h;
  h.template load<kConcSuffix>(t, p, *v);
  const uint32_t lk = klen - layer - 1u;
  if (h.klen != lk) return 0;
  return suffix_compare<T, kConcSuffix>(t, p, h, key + layer + 1u, lk).sign == 0 ? 1 : 0;
}

// ---- update -------------------------------------------------------------------------

template <int T>
MT_DEV int coop_update(const tile<T>& t, const tree_view& tv, slab_cache<T>& cache, const uint32_t* key,
                       uint32_t klen, const uint32_t* val, uint32_t vlen) {
  const pool_view& p = tv.pool;
  if (klen == 0u || vlen > kMaxLen16) {
    if (t.leader()) record_error(p, ERR_INVALID_ARG, MT_AT(SRC_TREE));
    return RES_ERR;
  }
  uint32_t root = tv.root, hops = 0;
  node<T> nd;
  for (uint32_t layer = 0; layer < klen;) {
    const uint32_t slice = key[layer];
    const bool more = layer + 1u < klen;
    if (!descend<T, kConc>(t, p, root, slice, nd, hops)) return RES_ERR;
    if (more) {
      const int e = nd.match(t, slice, true);
      if (e >= 0 && ks_get(nd.ks, (uint32_t)e) == KS_LINK) { root = nd.val_at(t, (uint32_t)e); ++layer; continue; }
    }
    uint32_t v0 = kInvalid;
    if (!present_in_image(t, p, nd, key, klen, layer, &v0)) return RES_FAIL;
    if (!lock_border(t, p, slice, nd, hops)) return RES_ERR;
    const int e = nd.match(t, slice, more);
    if (e < 0) { unlock_node(t, p, nd.idx); return RES_FAIL; }
    const uint32_t st = ks_get(nd.ks, (uint32_t)e);
    const uint32_t v = nd.val_at(t, (uint32_t)e);
    if (st == KS_LINK) { unlock_node(t, p, nd.idx); root = v; ++layer; continue; }
    if (st == KS_VALUE || st == KS_LONGVAL) return replace_value(t, p, cache, nd, (uint32_t)e, st, v, val, vlen);
    if (!p.valid(v)) { unlock_node(t, p, nd.idx); if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return RES_ERR; }
    const uint32_t lk = klen - layer - 1u;
    if (v != v0) {  // the chain changed since the lock-free check: compare again
      suffix_head<T> h;
      h.template load<kConcSuffix>(t, p, v);
      if (h.klen != lk || suffix_compare<T, kConcSuffix>(t, p, h, key + layer + 1u, lk).sign != 0) {
        unlock_node(t, p, nd.idx);
        return RES_FAIL;
      }
    }
    return replace_suffix(t, p, cache, nd, (uint32_t)e, v, key + layer + 1u, lk, val, vlen);
  }
  return RES_FAIL;
}

// ---- erase --------------------------------------------------------------------------

template <int T>
MT_DEV int coop_erase(const tile<T>& t, const tree_view& tv, const uint32_t* key, uint32_t klen) {
  const pool_view& p = tv.pool;
  if (klen == 0u) return RES_FAIL;
  uint32_t root = tv.root, hops = 0;
  node<T> nd;
  for (uint32_t layer = 0; layer < klen;) {
    const uint32_t slice = key[layer];
    const bool more = layer + 1u < klen;
    if (!descend<T, kConc>(t, p, root, slice, nd, hops)) return RES_ERR;
    if (more) {
      const int e = nd.match(t, slice, true);
      if (e >= 0 && ks_get(nd.ks, (uint32_t)e) == KS_LINK) { root = nd.val_at(t, (uint32_t)e); ++layer; continue; }
    }
    uint32_t v0 = kInvalid;
    if (!present_in_image(t, p, nd, key, klen, layer, &v0)) return RES_FAIL;
    if (!lock_border(t, p, slice, nd, hops)) return RES_ERR;
    const int e = nd.match(t, slice, more);
    if (e < 0) { unlock_node(t, p, nd.idx); return RES_FAIL; }
    const uint32_t st = ks_get(nd.ks, (uint32_t)e);
    const uint32_t v = nd.val_at(t, (uint32_t)e);
    if (st == KS_LINK) { unlock_node(t, p, nd.idx); root = v; ++layer; continue; }
    if (st == KS_SUFFIX && v != v0) {
      if (!p.valid(v)) { unlock_node(t, p, nd.idx); if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return RES_ERR; }
      suffix_head<T> h;
      h.template load<kConcSuffix>(t, p, v);
      const uint32_t lk = klen - layer - 1u;
      if (h.klen != lk || suffix_compare<T, kConcSuffix>(t, p, h, key + layer + 1u, lk).sign != 0) {
        unlock_node(t, p, nd.idx);
        return RES_FAIL;
      }
    }
    nd.remove_at(t, (uint32_t)e);
    publish_unlock(t, p, nd);
    if (st != KS_VALUE) suffix_retire<T, kConcSuffix>(t, p, v);
    if (tv.merge_log != nullptr && t.leader() && !nd.is_root() && (nd.count() == kMergeAt || nd.count() == 0u)) {
      const uint32_t r = atomicAdd(tv.merge_log, 1u);
      if (r < tv.merge_cap) {
        tv.merge_log[2u + 2u * r] = root;
        tv.merge_log[3u + 2u * r] = slice;
      }
    }
    // A layer's empty root is logged for removal; with merges also its emptied
    // rightmost border node, as the merges may fold the layer into its root.
    if (tv.layer_log != nullptr && t.leader() && layer >= 1u && layer < kLayerRecWords && nd.count() == 0u &&
        !nd.has_sib() && (nd.is_root() || tv.merge_log != nullptr)) {
      const uint32_t r = atomicAdd(tv.layer_log, 1u);
      if (r < tv.layer_cap) {
        uint32_t* rec = tv.layer_log + 2u + (size_t)kLayerRecWords * r;
        rec[0] = layer;
        for (uint32_t i = 0; i < layer; ++i) rec[1u + i] = key[i];
      }
    }
    return RES_OK;
  }
  return RES_FAIL;
}

// ---- scan ----------------------------------------------------------------------------

// Per-layer scan frame: border node holding the LINK we descended through,
// the LINK's slice, and whether the layer was on the upper bound's path.
struct scan_frame {
  uint32_t node;
  uint32_t slice;
  uint32_t upper_tight;
  uint32_t pad;
};

// The layer stack of one scan (the reference's tile-local dynamic_stack, which
// keeps 31 entries in registers and spills to slabs, include/dynamic_stack.hpp:
// 30-152).  Frames [0, fast_cap) live in a caller-provided global array; deeper
// frames spill to pool slabs of kFramesPerSlab frames each (frame k at words
// 4k..4k+3, word 31 = the slab below), taken from the tile's slab cache and
// retired when the stack shrinks or the scan ends.  Spill slabs are private to
// the tile.  Without a cache (and for fast_cap layers and more) a deeper scan
// reports MT_ERR_KEY_TOO_LONG.  Every member function is called by the whole
// tile; slice_at is per lane.
constexpr uint32_t kFramesPerSlab = 7;

template <int T>
struct scan_frames {
  scan_frame* fast = nullptr;
  uint32_t fast_cap = 0;
  slab_cache<T>* cache = nullptr;
  uint32_t cur = kInvalid;  // top spill slab (uniform)
  uint32_t base = 0;        // first spilled frame index (above fast_cap) held by `cur`

  MT_DEV scan_frames(scan_frame* f, uint32_t cap, slab_cache<T>* c) : fast(f), fast_cap(cap), cache(c) {}

  // Drop spill slabs until `cur` holds spilled frame i (or none are left).
  MT_DEV void shrink_to(const tile<T>& t, const pool_view& p, uint32_t i) {
    while (cur != kInvalid && i < base) {
      const uint32_t below = ld_word<ld_order::RELAXED>(p.addr(cur) + 31);
      t.sync();
      if (t.leader()) retire_slab(p, cur);
      cur = below;
      base = base >= kFramesPerSlab ? base - kFramesPerSlab : 0u;
    }
  }
  MT_DEV bool push(const tile<T>& t, const pool_view& p, uint32_t layer, const scan_frame& f) {
    if (layer < fast_cap) {
      if (t.leader()) fast[layer] = f;
      t.sync();
      return true;
    }
    const uint32_t i = layer - fast_cap;
    shrink_to(t, p, i);
    if (cur == kInvalid || i >= base + kFramesPerSlab) {
      if (cache == nullptr) {
        if (t.leader()) record_error(p, ERR_KEY_TOO_LONG, MT_AT(SRC_TREE));
        return false;
      }
      const uint32_t s = cache->allocate(t, p);
      if (s == kInvalid) return false;
      if (t.leader()) p.addr(s)[31] = cur;
      base = (cur == kInvalid) ? 0u : base + kFramesPerSlab;
      cur = s;
    }
    if (t.leader()) {
      uint32_t* w = p.addr(cur) + 4u * (i - base);
      w[0] = f.node;
      w[1] = f.slice;
      w[2] = f.upper_tight;
      w[3] = f.pad;
    }
    t.sync();
    return true;
  }
  // Frame `layer` after the stack shrank to it (frames above it are dropped).
  MT_DEV scan_frame pop_to(const tile<T>& t, const pool_view& p, uint32_t layer) {
    if (layer < fast_cap) {
      if (cur != kInvalid) release(t, p);
      return fast[layer];
    }
    const uint32_t i = layer - fast_cap;
    shrink_to(t, p, i);
    const uint32_t* w = p.addr(cur) + 4u * (i - base);
    scan_frame f;
    f.node = w[0];
    f.slice = w[1];
    f.upper_tight = w[2];
    f.pad = w[3];
    return f;
  }
  // LINK slice of frame i below the top of the stack (per lane).
  MT_DEV uint32_t slice_at(const pool_view& p, uint32_t i) const {
    if (i < fast_cap) return fast[i].slice;
    const uint32_t j = i - fast_cap;
    uint32_t s = cur, b = base;
    while (j < b && s != kInvalid) {
      s = p.addr(s)[31];
      b -= kFramesPerSlab;
    }
    return s == kInvalid ? 0u : p.addr(s)[4u * (j - b) + 1u];
  }
  // Retire every spill slab (the scan ended).
  MT_DEV void release(const tile<T>& t, const pool_view& p) {
    t.sync();
    if (t.leader()) {
      uint32_t c = cur;
      while (c != kInvalid) {
        const uint32_t below = p.addr(c)[31];
        retire_slab(p, c);
        c = below;
      }
    }
    cur = kInvalid;
    base = 0;
    t.sync();
  }
};

struct scan_out {
  uint32_t* values;
  uint32_t* value_lengths;
  uint32_t maxV;
  uint32_t* keys;
  uint32_t* key_lengths;
  uint32_t maxK;
};

// Emit one result: key = frames[0..layer) slices ++ slice ++ suffix rest.
template <int T, ld_order OS>
MT_DEV void scan_emit(const tile<T>& t, const pool_view& p, const scan_frames<T>& frames, uint32_t layer,
                      uint32_t slice, uint32_t state, uint32_t v, const suffix_head<T>* h,
                      const scan_out& o, uint32_t c) {
  uint32_t rest = 0, vlen = 1;
  if (state != KS_VALUE) { rest = h->klen; vlen = h->vlen; }
  const uint32_t klen = layer + 1u + rest;
  if (o.keys) {
    uint32_t* row = o.keys + (size_t)c * o.maxK;
    for (uint32_t i = t.rank; i < layer && i < o.maxK; i += T) row[i] = frames.slice_at(p, i);
    if (t.leader() && layer < o.maxK) row[layer] = slice;
    if (rest) {
      // Key rest: data slices [0, rest) of the chain.
      constexpr int W = 32 / T;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const uint32_t g = t.rank * W + q;
        if (g < kSufData && g < rest && layer + 1u + g < o.maxK) row[layer + 1u + g] = h->w[q];
      }
      for (uint32_t i = kSufData + t.rank; i < rest && layer + 1u + i < o.maxK; i += T)
        row[layer + 1u + i] = chain_slice<OS>(p, h->idx, i);
    }
  }
  if (o.key_lengths && t.leader()) o.key_lengths[c] = klen;
  if (o.value_lengths && t.leader()) o.value_lengths[c] = vlen;
  if (o.values && o.maxV > 0u) {
    uint32_t* vrow = o.values + (size_t)c * o.maxV;
    if (state == KS_VALUE) {
      if (t.leader()) vrow[0] = v;
    } else {
      suffix_get_value<T, OS>(t, p, *h, vrow, o.maxV);
    }
  }
}

// Ordered scan from `lower` (inclusive) for at most max_count keys, stopping
// after `upper` (inclusive) when use_upper.  frames: the tile's layer stack
// (empty on entry; emptied again on return).  Returns the number of keys
// written.
template <int T, bool CONCURRENT>
MT_DEV uint32_t coop_scan_walk(const tile<T>& t, const tree_view& tv, const uint32_t* lower, uint32_t llen,
                               bool use_upper, const uint32_t* upper, uint32_t ulen, uint32_t max_count,
                               const scan_out& o, scan_frames<T>& frames);

template <int T, bool CONCURRENT>
MT_DEV uint32_t coop_scan(const tile<T>& t, const tree_view& tv, const uint32_t* lower, uint32_t llen,
                          bool use_upper, const uint32_t* upper, uint32_t ulen, uint32_t max_count,
                          const scan_out& o, scan_frames<T>& frames) {
  const uint32_t c = coop_scan_walk<T, CONCURRENT>(t, tv, lower, llen, use_upper, upper, ulen, max_count, o, frames);
  if (frames.cur != kInvalid) frames.release(t, tv.pool);
  return c;
}

// Ask L2 for the lines a scan reads next in border node nd: the chain (or
// child layer root) of every entry from `start` on, and the right sibling.
// Each lane handles the entries whose value words it holds, so nothing is
// exchanged and no register stays busy: the scan still reads the lines one
// entry at a time, but from L2 instead of DRAM.
template <int T>
MT_DEV void prefetch_scan_lines(const tile<T>& t, const pool_view& p, const node<T>& nd, uint32_t start) {
  const uint32_t n = nd.count();
#pragma unroll
  for (int k = 0; k < node<T>::W; ++k) {
    const uint32_t g = t.rank * node<T>::W + (uint32_t)k;
    if ((g & 1u) == 0u || g >= 2u * (uint32_t)kMaxEntries) continue;
    const uint32_t e = g >> 1;
    if (e < start || e >= n || ks_get(nd.ks, e) == KS_VALUE || !p.valid(nd.w[k])) continue;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p.addr(nd.w[k])));
  }
  if (t.leader() && nd.has_sib() && p.valid(nd.sib)) asm volatile("prefetch.global.L2 [%0];" ::"l"(p.addr(nd.sib)));
}

template <int T, bool CONCURRENT>
MT_DEV uint32_t coop_scan_walk(const tile<T>& t, const tree_view& tv, const uint32_t* lower, uint32_t llen,
                               bool use_upper, const uint32_t* upper, uint32_t ulen, uint32_t max_count,
                               const scan_out& o, scan_frames<T>& frames) {
  constexpr ld_order O = CONCURRENT ? kConc : ld_order::NC;
  constexpr ld_order OS = CONCURRENT ? kConcSuffix : ld_order::NC;
  const pool_view& p = tv.pool;
  if (max_count == 0u) return 0u;
  if (use_upper && ulen == 0u) return 0u;
  uint32_t count = 0, hops = 0, layer = 0;
  const uint32_t hop_limit = kMaxHops + 8u * max_count;
  bool ltight = llen > 0u;   // still on the lower bound's path
  bool utight = use_upper;   // still on the upper bound's path
  node<T> nd;
  uint32_t start;
  // Enter layer 0.
  {
    const uint32_t s0 = ltight ? lower[0] : 0u;
    if (!descend<T, O>(t, p, tv.root, s0, nd, hops, hop_limit)) return 0u;
    start = ltight ? nd.lower_pos(t, s0, llen > 1u) : 0u;
  }
  while (true) {
    // Walk entries [start, count) of the border node nd at `layer`.
    bool descended = false;
    const uint32_t n = nd.count();
    prefetch_scan_lines(t, p, nd, start);
    for (uint32_t e = start; e < n; ++e) {
      const uint32_t s = nd.key_at(t, e);
      const uint32_t st = ks_get(nd.ks, e);
      const uint32_t v = nd.val_at(t, e);
      const bool more = ks_more(st);
      bool child_ltight = false;
      bool child_utight = false;
      suffix_head<T> h;
      const bool has_chain = st == KS_SUFFIX || st == KS_LONGVAL;
      if (has_chain) {
        if (!p.valid(v)) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return count; }
        h.template load<OS>(t, p, v);
      }
      if (ltight) {
        const uint32_t ls = lower[layer];
        const bool lm = layer + 1u < llen;
        if (pos_less(s, more, ls, lm)) continue;
        if (s == ls && more == lm) {
          if (st == KS_SUFFIX) {
            if (suffix_compare<T, OS>(t, p, h, lower + layer + 1u, llen - layer - 1u).sign < 0) continue;
          } else if (st == KS_LINK) {
            child_ltight = true;
          }
        }
        ltight = false;
      }
      if (utight) {
        const uint32_t us = upper[layer];
        const bool um = layer + 1u < ulen;
        if (pos_less(us, um, s, more)) return count;  // entry beyond upper
        if (s == us && more == um) {
          if (st == KS_SUFFIX) {
            if (suffix_compare<T, OS>(t, p, h, upper + layer + 1u, ulen - layer - 1u).sign > 0) return count;
          } else if (st == KS_LINK) {
            child_utight = true;
          }
        }
      }
      if (st == KS_LINK) {
        scan_frame f;
        f.node = nd.idx;
        f.slice = s;
        f.upper_tight = utight ? 1u : 0u;
        f.pad = 0u;
        if (!frames.push(t, p, layer, f)) return count;
        ++layer;
        ltight = child_ltight;
        utight = child_utight;
        const uint32_t s0 = ltight ? lower[layer] : 0u;
        if (!descend<T, O>(t, p, v, s0, nd, hops, hop_limit)) return count;
        start = ltight ? nd.lower_pos(t, s0, layer + 1u < llen) : 0u;
        descended = true;
        break;
      }
      scan_emit<T, OS>(t, p, frames, layer, s, st, v, has_chain ? &h : nullptr, o, count);
      ++count;
      if (count >= max_count) return count;
      if (utight && s == upper[layer] && more == (layer + 1u < ulen)) return count;  // emitted upper itself
    }
    if (descended) continue;
    ltight = false;
    // Next border node of this layer.
    if (nd.has_sib()) {
      if (utight && nd.high >= upper[layer]) return count;
      const uint32_t sib = nd.sib;
      if (!p.valid(sib) || ++hops > hop_limit) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return count; }
      if (!nd.template load_verified<O>(t, p, sib)) return count;
      start = 0;
      continue;
    }
    // End of this layer: resume the parent layer after the LINK slice.
    if (layer == 0u) return count;
    t.sync();
    --layer;
    const scan_frame f = frames.pop_to(t, p, layer);
    utight = f.upper_tight != 0u;
    if (utight && f.slice == upper[layer]) return count;  // the LINK was upper's own path
    if (f.slice == 0xFFFFFFFFu) {
      // Nothing can follow slice 0xFFFFFFFF in this layer.
      nd.meta = 0u;  // empty image: fall through to sibling/pop handling
      nd.idx = f.node;
      start = 0;
      continue;
    }
    if (!p.valid(f.node)) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return count; }
    if (!nd.template load_verified<O>(t, p, f.node)) return count;
    while (nd.must_move_right(f.slice)) {
      if (!p.valid(nd.sib) || ++hops > hop_limit) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return count; }
      if (!nd.template load_verified<O>(t, p, nd.sib)) return count;
    }
    start = __popc(nd.entry_mask(t, [&](uint32_t k, uint32_t) { return k <= f.slice; }));
  }
}

}  // namespace mtb
