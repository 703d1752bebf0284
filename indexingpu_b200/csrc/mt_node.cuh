// B-link tree node of one trie layer, held in registers by a tile.
//
// One node is one 128-byte slab = 32 u32 words:
//   entries 0..12 : word 2e = key slice, word 2e+1 = value
//                   border node  : value = inline value / suffix slab / layer root
//                   interior node: key = separator (largest slice routed to the
//                                  child), value = child slab
//   word 26       : checksum of the other 31 words (LOCK bit masked)
//   word 27       : reserved (0)
//   word 28       : high key (largest slice this node covers; 0xFFFFFFFF for the
//                   rightmost node of a level)
//   word 29       : right sibling slab (valid iff META_SIB)
//   word 30       : meta  = count:4 | LOCK | BORDER | SIB | ROOT | DEAD | version:16 (bits 16..31)
//   word 31       : keystates of a border node, 2 bits per entry
//
// Why a checksum: on B200 a 128-byte line stored by one warp instruction is
// NOT always observed atomically by a concurrent 128-byte load (the line
// self-test, mt_selftest_line_atomicity, counts torn reads at every tile width,
// about 1 in 10^5 reads under contention).  Lock-free readers therefore verify
// the checksum and reload on a mismatch; writers recompute it on every publish.
// The reference keeps the same defence behind a switch that is compiled out
// (include/compute_hash.hpp:179-199) and relies on atomicity instead.
//
// Keystate (bit0 = "key continues past this slice", bit1 = "value is a slab"):
//   VALUE 00 : key ends here, value is the inline u32 value (value length 1)
//   LINK  01 : key continues, value = root slab of the next trie layer
//   LONGVAL 10 : key ends here, value = suffix chain holding the value
//   SUFFIX  11 : key continues, value = suffix chain holding key rest + value
// These four states and their 2-bit encoding are the reference's entry kinds
// (include/masstree_node_subwarp.hpp:33-36, 968-994); the word placement,
// metadata packing and the 4..32-lane register layout are this library's own.
// A border node keeps entries sorted by (slice, continues) so that a key that
// ends at a slice sorts before one that continues with it (the reference's
// cmp_key, include/masstree_node_subwarp.hpp:312-314).
//
// Lane r of a tile of T lanes holds words [r*W, r*W+W), W = 32/T.
#pragma once
#include "mt_pool.cuh"

namespace mtb {

constexpr int kMaxEntries = 13;
constexpr uint32_t kTornRetries = 1u << 12;  // reloads of a torn node image before MT_ERR_CORRUPT
constexpr uint32_t KS_VALUE = 0u, KS_LINK = 1u, KS_LONGVAL = 2u, KS_SUFFIX = 3u;
constexpr uint32_t KS_MORE = 1u, KS_SLAB = 2u;

constexpr uint32_t META_COUNT = 0xFu;
constexpr uint32_t META_LOCK = 1u << 4;
constexpr uint32_t META_BORDER = 1u << 5;
constexpr uint32_t META_SIB = 1u << 6;
constexpr uint32_t META_ROOT = 1u << 7;
// Set on the last image of a node that a merge folded into another one: a pass
// that locks a node through a stale path sees that it no longer belongs to the
// tree.  (Nothing else reads it; the slab is reused only after the launch.)
constexpr uint32_t META_DEAD = 1u << 8;
constexpr uint32_t META_VERSION_ONE = 1u << 16;

constexpr int WORD_CSUM = 26, WORD_HIGH = 28, WORD_SIB = 29, WORD_META = 30, WORD_KS = 31;

// Contribution of word g (value v) to a node checksum: a bijection of v for
// every position (xor with a position constant, multiply by an odd constant,
// xor-shift), so a torn image differing from a published one in a single word
// always fails, and one differing in several words passes only if their mixed
// differences cancel exactly modulo 2^32.  (One multiply per word: the
// verification runs on every lock-free node load.)
MT_HD uint32_t csum_term(uint32_t g, uint32_t v) {
  if (g == (uint32_t)WORD_CSUM) return 0u;
  if (g == (uint32_t)WORD_META) v &= ~(1u << 4);  // LOCK bit changes without a republish
  const uint32_t x = (v ^ (g * 0x9E3779B9u) ^ 0x5BD1E995u) * 0x7FEB352Du;
  return x ^ (x >> 15);
}
// Host/device checksum of a full 32-word node image.
MT_HD uint32_t node_checksum(const uint32_t* w) {
  uint32_t h = 0;
  for (uint32_t g = 0; g < 32u; ++g) h += csum_term(g, w[g]);
  return h;
}

MT_HD uint32_t ks_get(uint32_t ks, uint32_t e) { return (ks >> (2u * e)) & 3u; }
MT_HD bool ks_more(uint32_t state) { return (state & KS_MORE) != 0u; }

// (s1, more1) < (s2, more2) in key order (a key ending at a slice sorts first).
MT_HD bool pos_less(uint32_t s1, bool m1, uint32_t s2, bool m2) {
  return s1 < s2 || (s1 == s2 && !m1 && m2);
}

MT_DEV uint32_t compress_even_bits(uint32_t x) {
  x &= 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0F0F0F0Fu;
  x = (x | (x >> 4)) & 0x00FF00FFu;
  x = (x | (x >> 8)) & 0x0000FFFFu;
  return x;
}

template <int T>
struct node {
  static constexpr int W = 32 / T;
  uint32_t w[W];
  uint32_t idx = kInvalid;
  // Uniform decoded header (valid after decode()).
  uint32_t meta = 0, ks = 0, high = 0, sib = kInvalid;

  // ---- word access -------------------------------------------------------
  MT_DEV uint32_t word(const tile<T>& t, uint32_t g) const {
    return t.shfl(reg_select(w, g % W), (int)(g / W));
  }
  MT_DEV void set_word(const tile<T>& t, uint32_t g, uint32_t v) {
    if (t.rank == g / W) reg_assign(w, g % W, v);
  }
  MT_DEV void decode(const tile<T>& t) {
    meta = word(t, WORD_META);
    ks = word(t, WORD_KS);
    high = word(t, WORD_HIGH);
    sib = word(t, WORD_SIB);
  }
  MT_DEV void encode_header(const tile<T>& t) {
    set_word(t, WORD_META, meta);
    set_word(t, WORD_KS, ks);
    set_word(t, WORD_HIGH, high);
    set_word(t, WORD_SIB, sib);
  }

  MT_DEV uint32_t count() const { return meta & META_COUNT; }
  MT_DEV bool is_border() const { return (meta & META_BORDER) != 0u; }
  MT_DEV bool is_root() const { return (meta & META_ROOT) != 0u; }
  MT_DEV bool has_sib() const { return (meta & META_SIB) != 0u; }
  MT_DEV bool locked() const { return (meta & META_LOCK) != 0u; }
  MT_DEV bool dead() const { return (meta & META_DEAD) != 0u; }
  MT_DEV bool full() const { return count() >= (uint32_t)kMaxEntries; }
  // B-link move-right test: the slice lies beyond this node.
  MT_DEV bool must_move_right(uint32_t slice) const { return has_sib() && slice > high; }

  // ---- load / store -------------------------------------------------------
  template <ld_order O>
  MT_DEV void load(const tile<T>& t, const pool_view& p, uint32_t i) {
    idx = i;
    load_words<W, O>(p.addr(i) + t.rank * W, w);
    decode(t);
  }
  // Store the whole line; all tile lanes' earlier writes become visible first.
  template <st_order O>
  MT_DEV void store(const tile<T>& t, const pool_view& p) {
    t.sync();
    store_words<W, O>(p.addr(idx) + t.rank * W, w);
  }
  MT_DEV void clear_words() {
#pragma unroll
    for (int k = 0; k < W; ++k) w[k] = 0u;
  }
  MT_DEV uint32_t tile_checksum(const tile<T>& t) const {
    uint32_t h = 0;
#pragma unroll
    for (int k = 0; k < W; ++k) h += csum_term(t.rank * W + k, w[k]);
    return t.add_all(h);
  }
  // Write the checksum word of the current image (call after encode_header).
  MT_DEV void seal(const tile<T>& t) { set_word(t, WORD_CSUM, tile_checksum(t)); }
  // Load an image that concurrent writers may be publishing: reload until the
  // checksum matches (bounded), else record corruption.
  template <ld_order O>
  MT_DEV bool load_verified(const tile<T>& t, const pool_view& p, uint32_t i) {
    for (uint32_t r = 0; r < kTornRetries; ++r) {
      load<O>(t, p, i);
      if constexpr (O == ld_order::NC) return true;
      if (tile_checksum(t) == word(t, WORD_CSUM)) return true;
    }
    if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_NODE));
    return false;
  }

  // ---- entry queries --------------------------------------------------------
  // Bit e set iff e < count and pred(key_e, e) holds.
  template <typename F>
  MT_DEV uint32_t entry_mask(const tile<T>& t, F pred) const {
    const uint32_t n = count();
    if constexpr (W >= 2) {
      constexpr int E = W / 2;
      uint32_t bits = 0;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const uint32_t e = t.rank * E + j;
        if (e < n && pred(w[2 * j], e)) bits |= 1u << e;
      }
      return t.or_all(bits);
    } else {
      const uint32_t e = t.rank >> 1;
      const bool p = ((t.rank & 1u) == 0u) && e < n && pred(w[0], e);
      return compress_even_bits(t.ballot(p));
    }
  }
  // Bit e set iff e < count and pred(value_e) holds.
  template <typename F>
  MT_DEV uint32_t value_mask(const tile<T>& t, F pred) const {
    const uint32_t n = count();
    if constexpr (W >= 2) {
      constexpr int E = W / 2;
      uint32_t bits = 0;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const uint32_t e = t.rank * E + j;
        if (e < n && pred(w[2 * j + 1])) bits |= 1u << e;
      }
      return t.or_all(bits);
    } else {
      const uint32_t e = t.rank >> 1;
      const bool p = ((t.rank & 1u) == 1u) && e < n && pred(w[0]);
      return compress_even_bits(t.ballot(p) >> 1);
    }
  }
  MT_DEV int child_slot_of(const tile<T>& t, uint32_t child) const {
    const uint32_t m = value_mask(t, [&](uint32_t v) { return v == child; });
    return m ? (__ffs(m) - 1) : -1;
  }
  MT_DEV uint32_t key_at(const tile<T>& t, uint32_t e) const { return word(t, 2u * e); }
  MT_DEV uint32_t val_at(const tile<T>& t, uint32_t e) const { return word(t, 2u * e + 1u); }

  // Interior node: child covering slice (first separator >= slice); -1 if none.
  MT_DEV int child_pos(const tile<T>& t, uint32_t slice) const {
    const uint32_t m = entry_mask(t, [&](uint32_t k, uint32_t) { return slice <= k; });
    return m ? (__ffs(m) - 1) : -1;
  }
  // Border node: entry matching (slice, continues); -1 if none.
  MT_DEV int match(const tile<T>& t, uint32_t slice, bool more) const {
    const uint32_t kss = ks;
    const uint32_t m = entry_mask(t, [&](uint32_t k, uint32_t e) {
      return k == slice && ks_more(ks_get(kss, e)) == more;
    });
    return m ? (__ffs(m) - 1) : -1;
  }
  // Border node: a LINK entry for slice exists.
  MT_DEV bool has_link(const tile<T>& t, uint32_t slice) const {
    const uint32_t kss = ks;
    return entry_mask(t, [&](uint32_t k, uint32_t e) { return k == slice && ks_get(kss, e) == KS_LINK; }) != 0u;
  }
  // Border node: number of entries ordered before (slice, more).
  MT_DEV uint32_t lower_pos(const tile<T>& t, uint32_t slice, bool more) const {
    const uint32_t kss = ks;
    return __popc(entry_mask(t, [&](uint32_t k, uint32_t e) {
      return pos_less(k, ks_more(ks_get(kss, e)), slice, more);
    }));
  }

  // ---- entry edits (registers only) -----------------------------------------
  // Insert (key, val, state) at position p, shifting entries p.. right by one.
  MT_DEV void insert_at(const tile<T>& t, uint32_t p, uint32_t key, uint32_t val, uint32_t state) {
    const uint32_t n = count();
    const uint32_t lo = 2u * p, hi = 2u * n + 2u;  // words [lo+2, hi) take old word g-2
    uint32_t prev[W];
    if constexpr (W >= 4) {
      const uint32_t a = t.shfl_up(w[W - 2], 1), b = t.shfl_up(w[W - 1], 1);
#pragma unroll
      for (int k = 0; k < W; ++k) prev[k] = (k >= 2) ? w[k - 2] : (k == 0 ? a : b);
    } else if constexpr (W == 2) {
      prev[0] = t.shfl_up(w[0], 1);
      prev[1] = t.shfl_up(w[1], 1);
    } else {
      prev[0] = t.shfl_up(w[0], 2);
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint32_t g = t.rank * W + k;
      if (g >= lo + 2u && g < hi) w[k] = prev[k];
      else if (g == lo) w[k] = key;
      else if (g == lo + 1u) w[k] = val;
    }
    const uint32_t lowmask = (p == 0u) ? 0u : ((1u << (2u * p)) - 1u);
    ks = ((ks & lowmask) | ((ks & ~lowmask) << 2) | (state << (2u * p))) & 0x0FFFFFFFu;
    meta = (meta & ~META_COUNT) | (n + 1u);
  }
  // Remove entry p, shifting entries p+1.. left by one.
  MT_DEV void remove_at(const tile<T>& t, uint32_t p) {
    const uint32_t n = count();
    const uint32_t lo = 2u * p, hi = 2u * n;  // words [lo, hi-2) take old word g+2
    uint32_t next[W];
    if constexpr (W >= 4) {
      const uint32_t a = t.shfl_down(w[0], 1), b = t.shfl_down(w[1], 1);
#pragma unroll
      for (int k = 0; k < W; ++k) next[k] = (k + 2 < W) ? w[k + 2] : (k == W - 2 ? a : b);
    } else if constexpr (W == 2) {
      next[0] = t.shfl_down(w[0], 1);
      next[1] = t.shfl_down(w[1], 1);
    } else {
      next[0] = t.shfl_down(w[0], 2);
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint32_t g = t.rank * W + k;
      if (g >= lo && g + 2u < hi) w[k] = next[k];
      else if (g + 2u >= hi && g < hi) w[k] = 0u;
    }
    const uint32_t lowmask = (p == 0u) ? 0u : ((1u << (2u * p)) - 1u);
    ks = ((ks & lowmask) | ((ks >> 2) & ~lowmask)) & 0x0FFFFFFFu;
    meta = (meta & ~META_COUNT) | (n - 1u);
  }
  MT_DEV void set_entry(const tile<T>& t, uint32_t e, uint32_t val, uint32_t state) {
    set_word(t, 2u * e + 1u, val);
    ks = (ks & ~(3u << (2u * e))) | (state << (2u * e));
  }

  // Copy entries [p, count) of src into entries [0, count-p) of this node.
  MT_DEV void take_upper_from(const tile<T>& t, const node& src, uint32_t p) {
    const uint32_t n = src.count();
    const uint32_t sh = 2u * p;
    const uint32_t lim = 2u * (n - p);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint32_t g = t.rank * W + k;
      const uint32_t srcg = g + sh;
      const uint32_t v = t.shfl(reg_select(src.w, (uint32_t)((k + sh) % W)), (int)((srcg / W) % T));
      w[k] = (g < lim) ? v : 0u;
    }
  }
  // Append the entries of src (all greater than this node's) after this
  // node's entries; the caller checks that both fit.
  MT_DEV void append_from(const tile<T>& t, const node& src) {
    const uint32_t a = count(), b = src.count();
    const uint32_t sh = 2u * a;  // word g takes src word g - sh
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint32_t g = t.rank * W + k;
      const uint32_t srcg = (g + 32u - sh) & 31u;
      const uint32_t v = t.shfl(reg_select(src.w, (uint32_t)((k + W - (int)(sh % W)) % W)), (int)(srcg / W));
      if (g >= sh && g < sh + 2u * b) w[k] = v;
    }
    ks = (ks | (src.ks << sh)) & 0x0FFFFFFFu;
    meta = (meta & ~META_COUNT) | (a + b);
  }
  // Keep entries [0, p): clear the entry words [2p, 26).
  MT_DEV void truncate(const tile<T>& t, uint32_t p) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint32_t g = t.rank * W + k;
      if (g >= 2u * p && g < (uint32_t)WORD_CSUM) w[k] = 0u;
    }
  }
};

}  // namespace mtb
