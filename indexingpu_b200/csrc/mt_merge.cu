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
//
// Removal of emptied trie layers (MT_FLAG_REMOVE_EMPTY_LAYERS; the reference's
// erase<do_remove_empty_root>, include/gpu_masstree.hpp:914-960).  An erase
// that leaves the only node of a layer (1 or deeper) without entries logs the
// key's slices above that layer.  After the call's erases (and merges) a pass
// follows those slices to the border node that holds the layer's LINK entry,
// locks it, locks the layer root, and when the root is still an empty border
// node without siblings removes the LINK entry and retires the root; a parent
// layer that this empties is removed in turn.  Locks are taken from the
// shallower layer to the deeper one, so records of one pass cannot deadlock.
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
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
      return false;
    }
    if (!nd.template load_verified<kConc>(t, p, idx)) return false;
    if (nd.must_move_right(slice)) { idx = nd.sib; continue; }
    if (nd.is_border()) return false;
    const int c = nd.child_pos(t, slice);
    const uint32_t ch = c < 0 ? kInvalid : nd.val_at(t, (uint32_t)c);
    if (!p.valid(ch)) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
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
        if (!p.valid(left) && t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
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
        if (!p.valid(right) && t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
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

// Remove the layer that record `rec` names, then every layer above it that the
// removal leaves without entries.
MT_DEV void remove_layers(const tile<32>& t, const tree_view& tv, const uint32_t* rec) {
  const pool_view& p = tv.pool;
  node<32> nd, cn;
  for (uint32_t depth = rec[0]; depth >= 1u && depth < kLayerRecWords; --depth) {
    // The root of layer depth-1, through the LINK entries of the slices above.
    uint32_t root = tv.root, hops = 0;
    for (uint32_t layer = 0; layer + 1u < depth; ++layer) {
      if (!descend<32, kConc>(t, p, root, rec[1u + layer], nd, hops)) return;
      const int e = nd.match(t, rec[1u + layer], true);
      if (e < 0 || ks_get(nd.ks, (uint32_t)e) != KS_LINK) return;  // removed by an earlier record
      root = nd.val_at(t, (uint32_t)e);
    }
    const uint32_t slice = rec[depth];
    if (!descend<32, kConc>(t, p, root, slice, nd, hops) || !lock_border(t, p, slice, nd, hops)) return;
    const int e = nd.match(t, slice, true);
    if (e < 0 || ks_get(nd.ks, (uint32_t)e) != KS_LINK) {
      unlock_node(t, p, nd.idx);
      return;
    }
    const uint32_t child = nd.val_at(t, (uint32_t)e);
    if (!p.valid(child) || !lock_load(t, p, child, cn)) {
      if (!p.valid(child) && t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
      unlock_node(t, p, nd.idx);
      return;
    }
    if (!cn.is_border() || !cn.is_root() || cn.has_sib() || cn.count() != 0u) {  // refilled or split since
      unlock_node(t, p, child);
      unlock_node(t, p, nd.idx);
      return;
    }
    nd.remove_at(t, (uint32_t)e);
    publish_unlock(t, p, nd);
    unlock_node(t, p, child);
    if (t.leader()) retire_slab(p, child);
    if (!nd.is_root() || nd.count() != 0u || nd.has_sib()) return;
  }
}

__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) remove_layers_kernel(tree_view tv,
                                                                                      const uint32_t* log,
                                                                                      uint32_t cap) {
  tile<32> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  const uint32_t n = min(log[0], cap);
  for (uint32_t r = tile_id; r < n; r += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    remove_layers(t, tv, log + 2u + (size_t)kLayerRecWords * r);
  }
}

constexpr uint32_t kLayerCap = 1u << 18;  // layer-log records per call (later ones are dropped)

// Creates a log on first use; false when it does not fit beside the slab pool.
bool ensure_log(uint32_t*& log, size_t words) {
  if (log) return true;
  if (cudaMalloc(reinterpret_cast<void**>(&log), words * sizeof(uint32_t)) == cudaSuccess) return true;
  cudaGetLastError();
  log = nullptr;
  return false;
}

}  // namespace

int host_merge_begin(mt_masstree* t, cudaStream_t s, uint32_t flags) {
  // A log that does not fit beside the slab pool leaves the call erasing
  // without that pass.
  if ((flags & MT_FLAG_MERGE) && ensure_log(t->merge_log, 2u + 2u * (size_t)kMergeCap)) {
    if (cudaMemsetAsync(t->merge_log, 0, 2u * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
    t->tv.merge_log = t->merge_log;
    t->tv.merge_cap = kMergeCap;
  }
  if ((flags & MT_FLAG_REMOVE_EMPTY_LAYERS) && ensure_log(t->layer_log, 2u + (size_t)kLayerRecWords * kLayerCap)) {
    if (cudaMemsetAsync(t->layer_log, 0, 2u * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
    t->tv.layer_log = t->layer_log;
    t->tv.layer_cap = kLayerCap;
  }
  return MT_OK;
}

int host_merge_end(mt_masstree* t, cudaStream_t s, int rc) {
  const bool merges = t->tv.merge_log != nullptr, layers = t->tv.layer_log != nullptr;
  t->tv.merge_log = nullptr;
  t->tv.merge_cap = 0;
  t->tv.layer_log = nullptr;
  t->tv.layer_cap = 0;
  if (rc != MT_OK) return rc;
  if (merges) merge_kernel<<<std::max(1, t->sms * 4), kBlock, 0, s>>>(t->tv, t->merge_log, kMergeCap);
  if (layers) remove_layers_kernel<<<std::max(1, t->sms * 4), kBlock, 0, s>>>(t->tv, t->layer_log, kLayerCap);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

}  // namespace mtb
