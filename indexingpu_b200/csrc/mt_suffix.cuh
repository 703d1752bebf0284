// Suffix chains: the rest of a key past its border slice plus its value.
//
// A chain is one or more 128-byte slabs.  Every slab carries 30 data slices
// (words 0..29); word 30 of the head slab is the header
// (key_rest_length | value_length << 16) and word 31 of every slab is the next
// slab (kInvalid at the end).  Data slice i of (key rest ++ value) lives in slab
// i / 30, word i % 30.  Chains are immutable once published: an update writes a
// new chain and retires the old one, so readers need no locks.
//
// Role and header packing follow the reference's suffix node
// (include/suffix_node_subwarp.hpp:696-708: chained 128-byte nodes, 16-bit key
// and value lengths in the head); the word placement here is this library's own.
#pragma once
#include "mt_node.cuh"

namespace mtb {

constexpr uint32_t kSufData = 30;
constexpr int SUF_WORD_HDR = 30, SUF_WORD_NEXT = 31;
constexpr uint32_t kMaxLen16 = 0xFFFFu;

MT_HD uint32_t suf_nodes(uint32_t klen, uint32_t vlen) {
  const uint32_t n = klen + vlen;
  return n == 0u ? 1u : (n + kSufData - 1u) / kSufData;
}

// Read data slice j of a chain (per lane; walks j/30 links).
template <ld_order O>
MT_DEV uint32_t chain_slice(const pool_view& p, uint32_t head, uint32_t j) {
  uint32_t s = head;
  uint32_t hops = j / kSufData;
  while (hops--) {
    const uint32_t nx = ld_word<O>(p.addr(s) + SUF_WORD_NEXT);
    if (!p.valid(nx)) return 0u;
    s = nx;
  }
  return ld_word<O>(p.addr(s) + (j % kSufData));
}

// Source of slices for a new chain: either plain arrays or an existing chain.
struct slice_src {
  const uint32_t* ptr = nullptr;  // plain array (request buffer)
  uint32_t chain = kInvalid;      // or existing chain head
  uint32_t offset = 0;            // data-slice offset inside that chain
  uint32_t len = 0;
  template <ld_order O>
  MT_DEV uint32_t get(const pool_view& p, uint32_t i) const {
    if (ptr) return ptr[i];
    return chain_slice<O>(p, chain, offset + i);
  }
};

// Allocate and write a chain holding key rest `k` and value `v`.
// Returns the head slab, or kInvalid on pool exhaustion (error recorded; any
// slab taken is retired).
template <int T, ld_order O>
MT_DEV uint32_t suffix_create(const tile<T>& t, const pool_view& p, slab_cache<T>& cache,
                              const slice_src& k, const slice_src& v) {
  constexpr int W = 32 / T;
  const uint32_t nn = suf_nodes(k.len, v.len);
  const uint32_t total = k.len + v.len;
  // The next slab is allocated before the current one is written, so every
  // slab is written once with its final link.
  const uint32_t head = cache.allocate(t, p);
  if (head == kInvalid) return kInvalid;
  uint32_t cur = head;
  for (uint32_t n = 0; n < nn; ++n) {
    uint32_t nxt = kInvalid;
    if (n + 1u < nn) {
      nxt = cache.allocate(t, p);
      if (nxt == kInvalid) {
        // Exhausted: retire slabs 0..n (0..n-1 are written and linked).
        t.sync();
        if (t.leader()) {
          uint32_t c = head;
          for (uint32_t q = 0; q < n && p.valid(c); ++q) {
            const uint32_t nx2 = ld_word<ld_order::RELAXED>(p.addr(c) + SUF_WORD_NEXT);
            retire_slab(p, c);
            c = nx2;
          }
          retire_slab(p, cur);
        }
        t.sync();
        return kInvalid;
      }
    }
    uint32_t w[W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const uint32_t g = t.rank * W + q;
      uint32_t val = 0u;
      if (g < kSufData) {
        const uint32_t di = n * kSufData + g;
        if (di < k.len) val = k.template get<O>(p, di);
        else if (di < total) val = v.template get<O>(p, di - k.len);
      } else if (g == (uint32_t)SUF_WORD_HDR) {
        val = (n == 0) ? ((k.len & kMaxLen16) | ((v.len & kMaxLen16) << 16)) : 0u;
      } else {
        val = nxt;
      }
      w[q] = val;
    }
    store_words<W, st_order::WEAK>(p.addr(cur) + t.rank * W, w);
    cur = nxt;
  }
  t.sync();
  return head;
}

// Loaded head of a chain.
template <int T>
struct suffix_head {
  static constexpr int W = 32 / T;
  uint32_t w[W];
  uint32_t idx = kInvalid;
  uint32_t klen = 0, vlen = 0, next = kInvalid;

  template <ld_order O>
  MT_DEV void load(const tile<T>& t, const pool_view& p, uint32_t i) {
    idx = i;
    load_words<W, O>(p.addr(i) + t.rank * W, w);
    const uint32_t hdr = t.shfl(reg_select(w, SUF_WORD_HDR % W), SUF_WORD_HDR / W);
    next = t.shfl(reg_select(w, SUF_WORD_NEXT % W), SUF_WORD_NEXT / W);
    klen = hdr & kMaxLen16;
    vlen = hdr >> 16;
  }
};

// Compare the stored key rest S (length ls) with K[0..lk).
// Returns f = index of the first differing slice (or min(ls, lk) if one is a
// prefix of the other) and the sign of S vs K.
struct cmp_result {
  uint32_t first_diff;
  int sign;  // <0: S < K, 0: equal, >0: S > K
};

template <int T, ld_order O>
MT_DEV cmp_result suffix_compare(const tile<T>& t, const pool_view& p, const suffix_head<T>& h,
                                 const uint32_t* K, uint32_t lk) {
  constexpr int W = 32 / T;
  const uint32_t ls = h.klen;
  const uint32_t m = min(ls, lk);
  uint32_t f = m;
  uint32_t sv = 0, kv = 0;
  // Head slab from registers.
  {
    uint32_t local = 0xFFFFFFFFu;
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const uint32_t g = t.rank * W + q;
      if (g < kSufData && g < m && local == 0xFFFFFFFFu) {
        if (h.w[q] != K[g]) local = g;
      }
    }
    f = min(f, t.min_all(local));
  }
  // Further slabs.
  uint32_t nx = h.next;
  for (uint32_t base = kSufData; f == m && base < m; base += kSufData) {
    if (!p.valid(nx)) break;
    uint32_t w[W];
    load_words<W, O>(p.addr(nx) + t.rank * W, w);
    uint32_t local = 0xFFFFFFFFu;
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const uint32_t g = t.rank * W + q;
      const uint32_t di = base + g;
      if (g < kSufData && di < m && local == 0xFFFFFFFFu) {
        if (w[q] != K[di]) local = di;
      }
    }
    f = min(f, t.min_all(local));
    nx = t.shfl(reg_select(w, SUF_WORD_NEXT % W), SUF_WORD_NEXT / W);
  }
  cmp_result r;
  r.first_diff = f;
  if (f < m) {
    sv = (f < kSufData) ? t.shfl(reg_select(h.w, f % W), (int)(f / W)) : chain_slice<O>(p, h.idx, f);
    kv = K[f];
    r.sign = sv < kv ? -1 : 1;
  } else {
    r.sign = ls < lk ? -1 : (ls > lk ? 1 : 0);
  }
  return r;
}

// Copy min(vlen, maxV) value slices to out (lane-parallel). Returns vlen.
template <int T, ld_order O>
MT_DEV uint32_t suffix_get_value(const tile<T>& t, const pool_view& p, const suffix_head<T>& h,
                                 uint32_t* out, uint32_t maxV) {
  constexpr int W = 32 / T;
  const uint32_t n = min(h.vlen, maxV);
  if (n == 0u || out == nullptr) return h.vlen;
  const uint32_t first = h.klen;            // data index of value slice 0
  const uint32_t last = first + n;          // exclusive
  // Slices inside the head slab come from registers.
#pragma unroll
  for (int q = 0; q < W; ++q) {
    const uint32_t g = t.rank * W + q;
    if (g < kSufData && g >= first && g < last) out[g - first] = h.w[q];
  }
  if (last > kSufData) {
    // Remaining slices: walk the chain slab by slab.
    uint32_t nx = h.next;
    for (uint32_t base = kSufData; base < last; base += kSufData) {
      if (!p.valid(nx)) break;
      uint32_t w[W];
      load_words<W, O>(p.addr(nx) + t.rank * W, w);
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const uint32_t g = t.rank * W + q;
        const uint32_t di = base + g;
        if (g < kSufData && di >= first && di < last) out[di - first] = w[q];
      }
      nx = t.shfl(reg_select(w, SUF_WORD_NEXT % W), SUF_WORD_NEXT / W);
    }
  }
  return h.vlen;
}

// Retire every slab of a chain (leader lane walks the links).
template <int T, ld_order O>
MT_DEV void suffix_retire(const tile<T>& t, const pool_view& p, uint32_t head) {
  if (t.leader() && p.valid(head)) {
    // Walk exactly the slabs the header accounts for, so that a damaged link
    // can never free slabs that belong to something else.
    const uint32_t hdr = ld_word<O>(p.addr(head) + SUF_WORD_HDR);
    const uint32_t nn = suf_nodes(hdr & kMaxLen16, hdr >> 16);
    uint32_t c = head;
    for (uint32_t q = 0; q < nn; ++q) {
      if (!p.valid(c)) { record_error(p, ERR_CORRUPT, MT_AT(SRC_SUFFIX)); break; }
      const uint32_t nx = ld_word<O>(p.addr(c) + SUF_WORD_NEXT);
      retire_slab(p, c);
      c = nx;
    }
    if (c != kInvalid) record_error(p, ERR_CORRUPT, MT_AT(SRC_SUFFIX));
  }
  t.sync();
}

}  // namespace mtb
