// TEST INFRASTRUCTURE ONLY.  C ABI over the reference's own gpu_masstree,
// compiled from the reference's headers where they lie (see oracle/Makefile).
// Used by the GPU parity tests as the primary oracle, and by
// `bench.py --impl reference` as the reference arm.  Instantiates exactly the
// configuration of the reference's evaluation adapter defaults
// (evaluation/gpu_masstree_adapter.hpp:173-180: tile 16, suffix on, merge level
// 4, lookup_concurrent off): gpu_masstree<simple_slab_allocator<128>,
// simple_debra_reclaimer<>, 16>, calling its public host API unchanged.
#include <cuda_runtime.h>

#include <cstdint>
#include <gpu_masstree.hpp>

namespace {
using alloc_t = simple_slab_allocator<128>;
using recl_t = simple_debra_reclaimer<>;
using tree_t = GpuMasstree::gpu_masstree<alloc_t, recl_t, 16>;

struct ref_tree {
  alloc_t alloc;
  recl_t recl;
  tree_t tree;
  explicit ref_tree(float ratio) : alloc(ratio), recl(), tree(alloc, recl) {}
};
}  // namespace

extern "C" {

void* ref_create(float pool_ratio) { return new ref_tree(pool_ratio); }

void ref_destroy(void* h) { delete static_cast<ref_tree*>(h); }

void ref_insert(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* vals,
                uint32_t maxV, const uint32_t* vlens, uint32_t n, void* stream) {
  static_cast<ref_tree*>(h)->tree.insert(keys, maxK, klens, vals, maxV, vlens, n, (cudaStream_t)stream);
}

void ref_update(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* vals,
                uint32_t maxV, const uint32_t* vlens, uint32_t n, void* stream) {
  static_cast<ref_tree*>(h)->tree.update(keys, maxK, klens, vals, maxV, vlens, n, (cudaStream_t)stream);
}

void ref_erase(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t n, void* stream) {
  static_cast<ref_tree*>(h)->tree.erase(keys, maxK, klens, n, (cudaStream_t)stream);
}

void ref_find(void* h, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t* vals, uint32_t maxV,
              uint32_t* vlens, uint32_t n, int concurrent, void* stream) {
  auto& t = static_cast<ref_tree*>(h)->tree;
  if (concurrent) t.find<true>(keys, maxK, klens, vals, maxV, vlens, n, (cudaStream_t)stream);
  else t.find<false>(keys, maxK, klens, vals, maxV, vlens, n, (cudaStream_t)stream);
}

void ref_mixed(void* h, const uint8_t* types, const uint32_t* keys, uint32_t maxK, const uint32_t* klens,
               uint32_t* vals, uint32_t maxV, uint32_t* vlens, bool* results, uint32_t n, void* stream) {
  static_cast<ref_tree*>(h)->tree.mixed_batch(reinterpret_cast<const kernels::request_type*>(types), keys, maxK,
                                              klens, vals, maxV, vlens, results, n, (cudaStream_t)stream);
}

void ref_scan(void* h, const uint32_t* lower, const uint32_t* lower_lens, uint32_t maxK, uint32_t max_count,
              uint32_t nq, const uint32_t* upper, const uint32_t* upper_lens, int use_upper, uint32_t* counts,
              uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint32_t* out_keys, uint32_t* out_klens,
              void* stream) {
  auto& t = static_cast<ref_tree*>(h)->tree;
  if (use_upper)
    t.scan<true, false>(lower, lower_lens, maxK, max_count, nq, upper, upper_lens, counts, vals, maxV, vlens, out_keys,
                        out_klens, (cudaStream_t)stream);
  else
    t.scan<false, false>(lower, lower_lens, maxK, max_count, nq, nullptr, nullptr, counts, vals, maxV, vlens,
                         out_keys, out_klens, (cudaStream_t)stream);
}

int ref_sync(void* stream) {
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

}  // extern "C"
