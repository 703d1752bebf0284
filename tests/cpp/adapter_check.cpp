// Drives include/universal_bench/gpu_masstree_adapter.hpp the way the reference's
// evaluation/universal_bench.cu drives its adapter (parse, print_args,
// initialize, insert, find, scan, update, erase, mixed_batch, print_stats,
// destroy, initialize again) and checks every result against a host model.
// Without a GPU only the argument checks run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <numeric>
#include <random>
#include <vector>

#include "universal_bench/gpu_masstree_adapter.hpp"

namespace {

int failures = 0;
void expect(bool ok, const char* what) {
  if (!ok && failures++ < 20) std::printf("mismatch: %s\n", what);
}

template <typename F>
bool throws(F&& f) {
  try {
    f();
  } catch (const std::invalid_argument&) {
    return true;
  }
  return false;
}

// A one-byte request type of the caller's own, as universal_bench passes
// kernels::request_type.
enum caller_request_type : uint8_t { c_insert = 0, c_erase = 1, c_find = 2, c_update = 3 };

template <typename T>
T* upload(const std::vector<T>& h) {
  T* d = nullptr;
  cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(T));
  cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}
template <typename T>
std::vector<T> download(const T* d, size_t n) {
  std::vector<T> h(n);
  cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
  return h;
}

using key_t_ = std::vector<uint32_t>;

}  // namespace

int main() {
  // ---- arguments (no GPU needed) ----
  {
    std::vector<std::string> args = {"bench", "-tile_size=32", "--merge_level=2", "-write_tile_size=16",
                                     "-lookup_concurrent=TRUE", "-allocator_pool_ratio=0.05", "-num_keys=100"};
    gpu_masstree_adapter a;
    a.parse(args);
    a.print_args();
    std::vector<std::string> bad_form = {"bench", "-tile_size"};
    std::vector<std::string> bad_tile = {"bench", "-tile_size=12"};
    std::vector<std::string> bad_merge = {"bench", "-merge_level=5"};
    std::vector<std::string> bad_ratio = {"bench", "-allocator_pool_ratio=0"};
    expect(throws([&] { gpu_masstree_adapter().parse(bad_form); }), "malformed argument rejected");
    expect(throws([&] { gpu_masstree_adapter().parse(bad_tile); }), "tile_size 12 rejected");
    expect(throws([&] { gpu_masstree_adapter().parse(bad_merge); }), "merge_level 5 rejected");
    expect(throws([&] { gpu_masstree_adapter().parse(bad_ratio); }), "pool ratio 0 rejected");
    bool logic = false;
    try {
      uint32_t k = 1;
      a.erase(&k, 1, nullptr, 1);
    } catch (const std::logic_error&) {
      logic = true;
    }
    expect(logic, "a call before initialize() throws");
  }
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
    std::printf("argument checks: %d mismatches; no GPU, device checks skipped\n", failures);
    return failures ? 1 : 0;
  }

  // ---- device calls ----
  // 70,000 keys: the first insert into the empty tree takes the bulk build for
  // keys whose first slice is unique and the ordinary insert for the rest.
  const uint32_t n = 70000, maxK = 4, maxV = 2, scan_count = 10, nscan = 500;
  std::mt19937 rng(11);
  std::vector<uint32_t> keys(n * maxK, 0), klens(n), vals(n * maxV, 0), vlens(n);
  std::map<key_t_, std::vector<uint32_t>> model;
  for (uint32_t i = 0; i < n; ++i) {
    for (;;) {
      klens[i] = 1 + rng() % maxK;
      key_t_ k(klens[i]);
      // First slices from 50,000 values spread over the u32 range (shared by
      // some keys, unique to others); later slices small (deeper layers).
      for (uint32_t j = 0; j < klens[i]; ++j) k[j] = j == 0 ? (rng() % 50000u) * 85899u : rng() % 64u;
      if (model.count(k)) continue;
      std::copy(k.begin(), k.end(), &keys[i * maxK]);
      vlens[i] = 1 + rng() % maxV;
      std::vector<uint32_t> v(vlens[i]);
      for (uint32_t s = 0; s < vlens[i]; ++s) v[s] = vals[i * maxV + s] = rng();
      model[k] = v;
      break;
    }
  }
  auto key_of = [&](uint32_t i) { return key_t_(&keys[i * maxK], &keys[i * maxK] + klens[i]); };

  std::vector<std::string> args = {"bench", "-tile_size=16", "-merge_level=4", "-allocator_pool_ratio=0.05",
                                   "-scan_tile_size=4"};
  gpu_masstree_adapter a;
  a.parse(args);
  a.initialize();
  uint32_t *dk = upload(keys), *dkl = upload(klens), *dv = upload(vals), *dvl = upload(vlens);
  uint32_t *ov = nullptr, *ovl = nullptr;
  cudaMalloc(&ov, (size_t)nscan * scan_count * maxV * 4 + n * maxV * 4);
  cudaMalloc(&ovl, (size_t)nscan * scan_count * 4 + n * 4);
  a.insert(dk, maxK, dkl, dv, maxV, dvl, n);

  auto check_finds = [&](const char* what) {
    cudaMemset(ovl, 0xFF, n * 4);
    a.find(dk, maxK, dkl, ov, maxV, ovl, n);
    expect(a.last_error() == MT_OK, "device error after find");
    auto gl = download(ovl, n);
    auto gv = download(ov, (size_t)n * maxV);
    for (uint32_t i = 0; i < n; ++i) {
      auto it = model.find(key_of(i));
      const uint32_t want = it == model.end() ? 0u : (uint32_t)it->second.size();
      bool ok = gl[i] == want;
      for (uint32_t s = 0; ok && s < want; ++s) ok = gv[(size_t)i * maxV + s] == it->second[s];
      expect(ok, what);
    }
  };
  check_finds("find after insert");

  // Scans of scan_count values from random lower bounds (present keys).
  {
    std::vector<uint32_t> lower(nscan * maxK, 0), llens(nscan);
    for (uint32_t q = 0; q < nscan; ++q) {
      const uint32_t i = rng() % n;
      std::copy(&keys[i * maxK], &keys[i * maxK] + maxK, &lower[q * maxK]);
      llens[q] = klens[i];
    }
    uint32_t *dl = upload(lower), *dll = upload(llens);
    cudaMemset(ovl, 0xFF, (size_t)nscan * scan_count * 4);
    a.scan(dl, maxK, dll, scan_count, ov, maxV, ovl, nscan, nullptr);
    expect(a.last_error() == MT_OK, "device error after scan");
    auto gl = download(ovl, (size_t)nscan * scan_count);
    auto gv = download(ov, (size_t)nscan * scan_count * maxV);
    for (uint32_t q = 0; q < nscan; ++q) {
      auto it = model.lower_bound(key_t_(&lower[q * maxK], &lower[q * maxK] + llens[q]));
      for (uint32_t r = 0; r < scan_count; ++r, ++it) {
        const size_t o = (size_t)q * scan_count + r;
        if (it == model.end()) break;
        bool ok = gl[o] == it->second.size();
        for (uint32_t s = 0; ok && s < it->second.size(); ++s) ok = gv[o * maxV + s] == it->second[s];
        expect(ok, "scan result");
      }
    }
    cudaFree(dl);
    cudaFree(dll);
  }

  // Update every second key, erase every third.
  {
    std::vector<uint32_t> uv(vals), uvl(vlens);
    for (uint32_t i = 0; i < n; i += 2) {
      uvl[i] = 1 + (i / 2) % maxV;
      std::vector<uint32_t> v(uvl[i]);
      for (uint32_t s = 0; s < uvl[i]; ++s) v[s] = uv[i * maxV + s] = 0xABC00000u + i * 2 + s;
      model[key_of(i)] = v;
    }
    // Only even requests carry new values: an update of an odd key writes its
    // unchanged value, which the model already holds.
    uint32_t *duv = upload(uv), *duvl = upload(uvl);
    a.update(dk, maxK, dkl, duv, maxV, duvl, n);
    check_finds("find after update");
    std::vector<uint32_t> ek, ekl;
    for (uint32_t i = 0; i < n; i += 3) {
      ek.insert(ek.end(), &keys[i * maxK], &keys[i * maxK] + maxK);
      ekl.push_back(klens[i]);
      model.erase(key_of(i));
    }
    uint32_t *dek = upload(ek), *dekl = upload(ekl);
    a.erase(dek, maxK, dekl, ekl.size());
    check_finds("find after erase");
    cudaFree(duv);
    cudaFree(duvl);
    cudaFree(dek);
    cudaFree(dekl);
  }

  // Mixed batch, every key once: keys i%4==0 erased (or re-inserted when
  // absent), 1 found, 2 updated, 3 found.
  {
    std::vector<caller_request_type> types(n);
    std::vector<uint32_t> mv(vals), mvl(vlens);
    std::vector<uint8_t> was_present(n);
    for (uint32_t i = 0; i < n; ++i) was_present[i] = model.count(key_of(i)) != 0;
    for (uint32_t i = 0; i < n; ++i) {
      const key_t_ k = key_of(i);
      switch (i % 4) {
        case 0:
          if (was_present[i]) {
            types[i] = c_erase;
            model.erase(k);
          } else {
            types[i] = c_insert;
            model[k] = std::vector<uint32_t>(&vals[i * maxV], &vals[i * maxV] + vlens[i]);
          }
          break;
        case 2:
          types[i] = c_update;
          mvl[i] = 2;
          mv[i * maxV] = 7 * i;
          mv[i * maxV + 1] = 7 * i + 1;
          if (was_present[i]) model[k] = {7 * i, 7 * i + 1};
          break;
        default:
          types[i] = c_find;
      }
    }
    auto dt = upload(types);
    uint32_t *dmv = upload(mv), *dmvl = upload(mvl);
    a.mixed_batch(dt, dk, maxK, dkl, dmv, maxV, dmvl, n);
    expect(a.last_error() == MT_OK, "device error after mixed batch");
    auto gl = download(dmvl, n);
    auto gv = download(dmv, (size_t)n * maxV);
    for (uint32_t i = 1; i < n; i += 2) {
      // Finds see the state before or after the batch's other requests on
      // other keys; their own key is touched once, so the model is exact.
      auto it = model.find(key_of(i));
      const uint32_t want = it == model.end() ? 0u : (uint32_t)it->second.size();
      bool ok = gl[i] == want;
      for (uint32_t s = 0; ok && s < want; ++s) ok = gv[(size_t)i * maxV + s] == it->second[s];
      expect(ok, "mixed-batch find");
    }
    check_finds("find after mixed batch");
    cudaFree(dt);
    cudaFree(dmv);
    cudaFree(dmvl);
  }

  std::string report;
  expect(a.index()->validate(&report), "validate");
  a.print_stats();
  a.destroy();

  // The universal bench initializes again for every phase: a fresh, empty tree.
  a.initialize();
  model.clear();
  check_finds("find on a re-initialized tree");
  a.print_stats();
  a.destroy();

  cudaFree(dk);
  cudaFree(dkl);
  cudaFree(dv);
  cudaFree(dvl);
  cudaFree(ov);
  cudaFree(ovl);
  std::printf("adapter: %d mismatches\n", failures);
  return failures ? 1 : 0;
}
