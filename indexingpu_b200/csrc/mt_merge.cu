// Merges of sparse border nodes after a call's erases (MT_FLAG_MERGE).
//
// The reference merges or borrows on the way down inside every erase
// (merge levels 2-4 of erase<>, include/gpu_masstree.hpp:751-971), holding up
// to three locks per request.  Here erases stay as they are; each erase that
// leaves a non-root border node with kMergeAt entries (or none) logs the node's
// layer root and slice, and after the call's erase kernels a pass runs over the
// log while nothing else works on the tree (calls on one tree do not overlap).
// For each logged node the pass locks its parent, then folds the node into its
// left neighbour under that parent, or its right neighbour into it, when the
// entries of both fit in one node; the emptied slab goes to the limbo list.
// Child 0 of a parent is never the slab given up, so the sibling links that
// cross parents stay valid.  Results never change, only space: a node merged
// away holds no key that its neighbour does not now hold.
#include <algorithm>

#include "mt_internal.cuh"

namespace mtb {
namespace {

constexpr uint32_t kMergeCap = 1u << 22;  // log records per call (later ones are dropped)

// The parent of the border node covering `slice` in the layer rooted at `root`,
// and that node.  False for a layer that is one border node (or on an error,
// which is recorded).
MT_DEV bool find_parent(const tile<32>& t, const pool_view& p, uint32_t root, uint32_t slice, uint32_t& parent,
                        uint32_t& child) {
  node<32> nd, cn;
  uint32_t idx = root, hops = 0;
  while (true) {
    if (!p.valid(idx) || ++hops > kMaxHops) {
      if (t.leader()) record_error(p, ERR_CORRUPT);
      return false;
    }
    if (!nd.template load_verified<kConc>(t, p, idx)) return false;
    if (nd.must_move_right(slice)) { idx = nd.sib; continue; }
    if (nd.is_border()) return false;
    const int c = nd.child_pos(t, slice);
    const uint32_t ch = c < 0 ? kInvalid : nd.val_at(t, (uint32_t)c);
    if (!p.valid(ch)) {
      if (t.leader()) record_error(p, ERR_CORRUPT);
      return false;
    }
    if (!cn.template load_verified<kConc>(t, p, ch)) return false;
    if (cn.is_border()) {
      parent = idx;
      child = ch;
      return true;
    }
    idx = ch;
  }
}

// dst takes src's entries after its own, and src's range, high key and sibling.
MT_DEV void absorb(const tile<32>& t, node<32>& dst, const node<32>& src) {
  dst.append_from(t, src);
  dst.high = src.high;
  dst.sib = src.sib;
  dst.meta = (dst.meta & ~META_SIB) | (src.meta & META_SIB);
}

MT_DEV void merge_one(const tile<32>& t, const pool_view& p, uint32_t root, uint32_t slice) {
  uint32_t parent = kInvalid, child = kInvalid;
  if (!find_parent(t, p, root, slice, parent, child)) return;
  node<32> pn, b, a;
  if (!lock_load(t, p, parent, pn)) return;
  const int i = pn.is_border() ? -1 : pn.child_slot_of(t, child);
  if (i < 0) {  // merged away by an earlier record
    unlock_node(t, p, parent);
    return;
  }
  const uint32_t n = pn.count();
  if (!p.valid(child) || !lock_load(t, p, child, b)) {
    unlock_node(t, p, parent);
    return;
  }
  if (b.is_border() && b.count() <= kMergeAt) {
    // Into the left neighbour: the parent's entry i-1 goes, entry i (the
    // separator of b's range) now routes to the neighbour.
    if (i >= 1) {
      const uint32_t left = pn.val_at(t, (uint32_t)i - 1u);
      if (!p.valid(left) || !lock_load(t, p, left, a)) {
        if (!p.valid(left) && t.leader()) record_error(p, ERR_CORRUPT);
        unlock_node(t, p, child);
        unlock_node(t, p, parent);
        return;
      }
      if (a.count() + b.count() <= (uint32_t)kMaxEntries) {
        absorb(t, a, b);
        publish_unlock(t, p, a);
        pn.remove_at(t, (uint32_t)i - 1u);
        pn.set_entry(t, (uint32_t)i - 1u, left, 0u);
        publish_unlock(t, p, pn);
        unlock_node(t, p, child);
        if (t.leader()) retire_slab(p, child);
        return;
      }
      unlock_node(t, p, left);
    }
    // Else the right neighbour into b: entry i goes, entry i+1 routes to b.
    if ((uint32_t)i + 1u < n) {
      const uint32_t right = pn.val_at(t, (uint32_t)i + 1u);
      if (!p.valid(right) || !lock_load(t, p, right, a)) {
        if (!p.valid(right) && t.leader()) record_error(p, ERR_CORRUPT);
        unlock_node(t, p, child);
        unlock_node(t, p, parent);
        return;
      }
      if (a.count() + b.count() <= (uint32_t)kMaxEntries) {
        absorb(t, b, a);
        publish_unlock(t, p, b);
        pn.remove_at(t, (uint32_t)i);
        pn.set_entry(t, (uint32_t)i, child, 0u);
        publish_unlock(t, p, pn);
        unlock_node(t, p, right);
        if (t.leader()) retire_slab(p, right);
        return;
      }
      unlock_node(t, p, right);
    }
  }
  unlock_node(t, p, child);
  unlock_node(t, p, parent);
}

__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) merge_kernel(tree_view tv, const uint32_t* log,
                                                                              uint32_t cap) {
  tile<32> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  const uint32_t n = min(log[0], cap);
  for (uint32_t r = tile_id; r < n; r += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    merge_one(t, tv.pool, log[2u + 2u * r], log[3u + 2u * r]);
  }
}

}  // namespace

int host_merge_begin(mt_masstree* t, cudaStream_t s) {
  if (!t->merge_log) {
    if (cudaMalloc(reinterpret_cast<void**>(&t->merge_log), (2u + 2u * (size_t)kMergeCap) * sizeof(uint32_t)) !=
        cudaSuccess) {
      // No room beside the slab pool: the call erases without merging.
      cudaGetLastError();
      t->merge_log = nullptr;
      return MT_OK;
    }
  }
  if (cudaMemsetAsync(t->merge_log, 0, 2u * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
  t->tv.merge_log = t->merge_log;
  t->tv.merge_cap = kMergeCap;
  return MT_OK;
}

int host_merge_end(mt_masstree* t, cudaStream_t s, int rc) {
  const bool logged = t->tv.merge_log != nullptr;
  t->tv.merge_log = nullptr;
  t->tv.merge_cap = 0;
  if (rc != MT_OK || !logged) return rc;
  merge_kernel<<<std::max(1, t->sms * 4), kBlock, 0, s>>>(t->tv, t->merge_log, kMergeCap);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

}  // namespace mtb
