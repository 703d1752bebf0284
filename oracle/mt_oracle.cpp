// TEST INFRASTRUCTURE ONLY — the oracle.  Nothing in the product links or calls
// this file; only tests/, the smoke check and bench.py's CPU-baseline leg do.
//
// CPU restatement of the observable semantics of IndexinGPU's gpu_masstree host
// API (include/gpu_masstree.hpp:86-191 of the reference):
//   * keys are u32 slice strings ordered lexicographically by slice value, a
//     key that is a prefix of another sorting first (the node order of
//     include/masstree_node_subwarp.hpp:312-314 plus suffix strcmp,
//     include/suffix_node_subwarp.hpp:112-186; the reference test sorts its
//     expected output with std::lexicographical_compare,
//     test/unittest_masstree.cu:153-159);
//   * find writes min(value_length, max_value_length) slices and returns the
//     full value length, 0 on a miss (gpu_masstree.hpp:194-248);
//   * insert does not overwrite unless update_if_exists (gpu_masstree.hpp:509-512);
//   * update fails on a miss (gpu_masstree.hpp:678-681); erase reports presence;
//   * scan returns the first max_count keys >= lower, stopping after upper when
//     given (both inclusive; test/unittest_masstree.cu:250-265 expects
//     end - begin + 1 results);
//   * mixed_batch requests run in index order (one valid linearisation of the
//     reference's unordered batch), request kinds 0 insert, 1 erase, 2 find,
//     3 update (include/macros.hpp:51-57).
// A sharded variant range-partitions the key space by the first slice and runs
// one thread per shard; it is the multi-core CPU baseline.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace {

using slices = std::u32string;  // char32_t compares as unsigned 32-bit

struct shard_map {
  std::map<slices, slices> m;
};

struct oracle {
  std::vector<shard_map> shards;
  uint32_t nshards = 1;
  uint32_t shard_of(const slices& k) const {
    if (nshards == 1 || k.empty()) return 0;
    return (uint32_t)(((uint64_t)(uint32_t)k[0] * nshards) >> 32);
  }
};

slices make_key(const uint32_t* keys, uint32_t maxK, const uint32_t* lens, uint32_t i) {
  const uint32_t l = lens ? lens[i] : maxK;
  const uint32_t* p = keys + (size_t)i * maxK;
  return slices(reinterpret_cast<const char32_t*>(p), l);
}

slices make_val(const uint32_t* vals, uint32_t maxV, const uint32_t* lens, uint32_t i) {
  const uint32_t l = lens ? lens[i] : maxV;
  const uint32_t* p = vals + (size_t)i * maxV;
  return slices(reinterpret_cast<const char32_t*>(p), l);
}

// One request against one map.  kind: 0 insert, 1 erase, 2 find, 3 update, 4 upsert.
void apply(std::map<slices, slices>& m, uint32_t kind, const slices& k, const uint32_t* vals, uint32_t maxV,
           const uint32_t* vlens_in, uint32_t* out_vals, uint32_t* out_vlens, uint8_t* results, uint32_t i) {
  switch (kind) {
    case 0: {
      auto r = m.emplace(k, make_val(vals, maxV, vlens_in, i));
      if (results) results[i] = r.second ? 1 : 0;
      break;
    }
    case 4: {
      m[k] = make_val(vals, maxV, vlens_in, i);
      if (results) results[i] = 1;
      break;
    }
    case 1: {
      const bool had = m.erase(k) > 0;
      if (results) results[i] = had ? 1 : 0;
      break;
    }
    case 3: {
      auto it = m.find(k);
      if (it != m.end()) it->second = make_val(vals, maxV, vlens_in, i);
      if (results) results[i] = it != m.end() ? 1 : 0;
      break;
    }
    default: {
      auto it = m.find(k);
      uint32_t l = 0;
      if (it != m.end()) {
        l = (uint32_t)it->second.size();
        const uint32_t c = std::min(l, maxV);
        if (out_vals) std::memcpy(out_vals + (size_t)i * maxV, it->second.data(), c * sizeof(uint32_t));
      }
      if (out_vlens) out_vlens[i] = l;
      break;
    }
  }
}

// Run n requests: each shard thread takes the requests whose key it owns, in
// index order.
void run(oracle* o, const uint8_t* kinds, uint32_t fixed_kind, const uint32_t* keys, uint32_t maxK,
         const uint32_t* klens, const uint32_t* vals, uint32_t maxV, const uint32_t* vlens_in, uint32_t* out_vals,
         uint32_t* out_vlens, uint8_t* results, uint32_t n, uint32_t threads) {
  auto body = [&](uint32_t s) {
    auto& m = o->shards[s].m;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t kl = klens ? klens[i] : maxK;
      const uint32_t first = kl ? keys[(size_t)i * maxK] : 0u;
      if (o->nshards > 1 && kl && (uint32_t)(((uint64_t)first * o->nshards) >> 32) != s) continue;
      if (o->nshards > 1 && !kl && s != 0) continue;
      const uint32_t kind = kinds ? kinds[i] : fixed_kind;
      apply(m, kind, make_key(keys, maxK, klens, i), vals, maxV, vlens_in, out_vals, out_vlens, results, i);
    }
  };
  if (o->nshards == 1 || threads <= 1) {
    for (uint32_t s = 0; s < o->nshards; ++s) body(s);
    return;
  }
  std::vector<std::thread> pool;
  for (uint32_t s = 0; s < o->nshards; ++s) pool.emplace_back(body, s);
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

void* oracle_create(uint32_t nshards) {
  auto* o = new oracle();
  o->nshards = nshards ? nshards : 1;
  o->shards.resize(o->nshards);
  return o;
}

void oracle_destroy(void* h) { delete static_cast<oracle*>(h); }

uint64_t oracle_size(void* h) {
  auto* o = static_cast<oracle*>(h);
  uint64_t n = 0;
  for (auto& s : o->shards) n += s.m.size();
  return n;
}

void oracle_insert(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* vals,
                   uint32_t maxV, const uint32_t* vlens, uint32_t n, uint8_t* results, int upsert, uint32_t threads) {
  run(static_cast<oracle*>(h), nullptr, upsert ? 4u : 0u, keys, maxK, klens, vals, maxV, vlens, nullptr, nullptr,
      results, n, threads);
}

void oracle_update(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* vals,
                   uint32_t maxV, const uint32_t* vlens, uint32_t n, uint8_t* results, uint32_t threads) {
  run(static_cast<oracle*>(h), nullptr, 3u, keys, maxK, klens, vals, maxV, vlens, nullptr, nullptr, results, n,
      threads);
}

void oracle_erase(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t n, uint8_t* results,
                  uint32_t threads) {
  run(static_cast<oracle*>(h), nullptr, 1u, keys, maxK, klens, nullptr, 0, nullptr, nullptr, nullptr, results, n,
      threads);
}

void oracle_find(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t* vals, uint32_t maxV,
                 uint32_t* vlens, uint32_t n, uint32_t threads) {
  run(static_cast<oracle*>(h), nullptr, 2u, keys, maxK, klens, nullptr, maxV, nullptr, vals, vlens, nullptr, n,
      threads);
}

void oracle_mixed(void* h, const uint8_t* kinds, const uint32_t* keys, uint32_t maxK, const uint32_t* klens,
                  uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint8_t* results, uint32_t n, uint32_t threads) {
  // vals / vlens are inputs for insert and update and outputs for find; the
  // inputs of request i are read before any output of request i is written.
  run(static_cast<oracle*>(h), kinds, 0u, keys, maxK, klens, vals, maxV, vlens, vals, vlens, results, n, threads);
}

// Ordered scan.  use_upper != 0 bounds the range by upper (inclusive).
void oracle_scan(void* h, const uint32_t* lower, const uint32_t* lower_lens, uint32_t maxK, uint32_t max_count,
                 uint32_t nq, const uint32_t* upper, const uint32_t* upper_lens, int use_upper, uint32_t* counts,
                 uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint32_t* out_keys, uint32_t* out_klens) {
  auto* o = static_cast<oracle*>(h);
  for (uint32_t q = 0; q < nq; ++q) {
    const slices lo = make_key(lower, maxK, lower_lens, q);
    slices up;
    if (use_upper) up = make_key(upper, maxK, upper_lens, q);
    uint32_t c = 0;
    for (uint32_t s = o->shard_of(lo); s < o->nshards && c < max_count; ++s) {
      auto& m = o->shards[s].m;
      for (auto it = m.lower_bound(lo); it != m.end() && c < max_count; ++it) {
        if (use_upper && up < it->first) { s = o->nshards; break; }
        const size_t slot = (size_t)q * max_count + c;
        const uint32_t kl = (uint32_t)it->first.size(), vl = (uint32_t)it->second.size();
        if (vlens) vlens[slot] = vl;
        if (vals) std::memcpy(vals + slot * maxV, it->second.data(), std::min(vl, maxV) * sizeof(uint32_t));
        if (out_klens) out_klens[slot] = kl;
        if (out_keys) std::memcpy(out_keys + slot * maxK, it->first.data(), std::min(kl, maxK) * sizeof(uint32_t));
        ++c;
      }
    }
    if (counts) counts[q] = c;
  }
}

// Dump every key in order (caller sizes the buffers with oracle_size).
void oracle_dump(void* h, uint32_t* keys, uint32_t maxK, uint32_t* klens, uint32_t* vals, uint32_t maxV,
                 uint32_t* vlens) {
  auto* o = static_cast<oracle*>(h);
  size_t i = 0;
  for (auto& s : o->shards) {
    for (auto& kv : s.m) {
      const uint32_t kl = (uint32_t)kv.first.size(), vl = (uint32_t)kv.second.size();
      klens[i] = kl;
      vlens[i] = vl;
      std::memcpy(keys + i * maxK, kv.first.data(), std::min(kl, maxK) * sizeof(uint32_t));
      std::memcpy(vals + i * maxV, kv.second.data(), std::min(vl, maxV) * sizeof(uint32_t));
      ++i;
    }
  }
}

}  // extern "C"
