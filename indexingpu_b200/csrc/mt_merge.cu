// Merges of sparse nodes after a call's erases (MT_FLAG_MERGE).
//
// The reference merges or borrows on the way down inside every erase
// (merge levels 2-4 of erase<>, include/gpu_masstree.hpp:751-971, with
// coop_traverse_until_border_merge, :1151-1350), holding up to three locks per
// request and node.  Here erases stay as they are; each erase that leaves a
// non-root border node with kMergeAt entries (or none) logs the node's layer
// root and slice, and after the call's erase kernels a pass runs over the log
// while nothing else works on the tree (calls on one tree do not overlap).
// For each logged node the pass walks the layer from its root and, from the
// border node upwards:
//   * locks the node's parent and the node, and when the node holds kMergeAt
//     entries or fewer folds it into its left neighbour under that parent, or
//     the right neighbour into it, when the entries of both fit in one node
//     (border and interior nodes alike: an interior entry is a separator and a
//     child, so two neighbours concatenate);
//   * goes on with the parent when that left it with kMergeAt entries or
//     fewer;
//   * when the parent is the layer root and has one child left, copies the
//     child into the root slab (the root keeps its slab, as the LINK entry
//     above and tree_view.root point to it), which takes one level off the
//     layer (the reference's merge_to_root, masstree_node_subwarp.hpp).
// Borrowing from a neighbour that does not fit (the reference's borrow_left /
// borrow_right) is not done: it keeps nodes fuller, it frees no slab.
// Child 0 of a parent is never the slab given up, so the sibling links that
// cross parents stay valid.  A node given up is republished with META_DEAD
// before it is retired: records work concurrently, and one that locks a node
// through a path read before the merge sees the flag and walks again.  Locks
// go from parent to child and, between neighbours, only under their parent's
// lock, so the pass cannot deadlock.  Results never change, only space: a node
// merged away holds no key that its neighbour does not now hold.
//
// Removal of emptied trie layers (MT_FLAG_REMOVE_EMPTY_LAYERS; the reference's
// erase<do_remove_empty_root>, include/gpu_masstree.hpp:914-960).  An erase
// that leaves a node of a layer (1 or deeper) without entries logs the key's
// slices above that layer: the layer's root when it is that node, any emptied
// node when merges run too (they may fold the layer back into an empty root).
// After the call's erases and merges a pass follows those slices to the border
// node that holds the layer's LINK entry, locks it, locks the layer root, and
// when the root is an empty border node without siblings removes the LINK
// entry and retires the root.  A parent layer that this empties is removed in
// turn; with merges, the border node that lost the LINK entry is merged
// upwards first.  Locks are taken from the shallower layer to the deeper one,
// so records of one pass cannot deadlock.
#include <algorithm>

#include "mt_internal.cuh"

namespace mtb {
namespace {

constexpr uint32_t kMergeCap = 1u << 22;  // log records per call (later ones are dropped)

constexpr uint32_t kMaxPath = 24;      // levels of one layer a merge walk follows (deeper: no merges)
constexpr uint32_t kMergeWalks = 8;    // walks from the root per record (a stale path costs one)

// The nodes from `root` down to the border node covering `slice` (after moves
// right), in path[0 .. n).  False on an error (recorded) or a layer deeper
// than kMaxPath.
struct merge_path {
  uint32_t n;
  uint32_t idx[kMaxPath];
};
MT_DEV bool walk_path(const tile<32>& t, const pool_view& p, uint32_t root, uint32_t slice, merge_path& mp) {
  node<32> nd;
  uint32_t idx = root, hops = 0;
  mp.n = 0;
  while (true) {
    if (!p.valid(idx) || ++hops > kMaxHops) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
      return false;
    }
    if (!nd.template load_verified<kConc>(t, p, idx)) return false;
    if (nd.must_move_right(slice)) { idx = nd.sib; continue; }
    if (mp.n == kMaxPath) return false;
    mp.idx[mp.n++] = idx;
    if (nd.is_border()) return true;
    const int c = nd.child_pos(t, slice);
    if (c < 0) {
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
      return false;
    }
    idx = nd.val_at(t, (uint32_t)c);
  }
}

// dst takes src's entries after its own, and src's range, high key and sibling.
MT_DEV void absorb(const tile<32>& t, node<32>& dst, const node<32>& src) {
  dst.append_from(t, src);
  dst.high = src.high;
  dst.sib = src.sib;
  dst.meta = (dst.meta & ~META_SIB) | (src.meta & META_SIB);
}

// Publish the last image of a node given up by a merge (flagged dead), release
// it and retire its slab.
MT_DEV void give_up(const tile<32>& t, const pool_view& p, node<32>& nd) {
  nd.meta |= META_DEAD;
  publish_unlock(t, p, nd);
  if (t.leader()) retire_slab(p, nd.idx);
}

// Lock a node a merge found through its parent (locked) or a walk; false, with
// nothing locked, when the lock fails (error recorded) or the node is dead.
MT_DEV bool lock_live(const tile<32>& t, const pool_view& p, uint32_t idx, node<32>& nd) {
  if (!p.valid(idx)) {
    if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
    return false;
  }
  if (!lock_load(t, p, idx, nd)) return false;
  if (nd.dead()) {
    unlock_node(t, p, idx);
    return false;
  }
  return true;
}

enum merge_step_result { STEP_ERROR, STEP_MERGED, STEP_KEPT, STEP_WALK };

// One merge under `parent`: node x (a border node iff `border`) with one of its
// neighbours, when x holds kMergeAt entries or fewer and both fit in one node.
// STEP_MERGED / STEP_KEPT (x merged / left as it is): *parent_count and
// *parent_root describe the parent afterwards.  STEP_WALK: the path was stale
// (a node dead or moved); walk again.  STEP_ERROR: a lock failed (recorded).
MT_DEV int merge_step(const tile<32>& t, const pool_view& p, uint32_t parent, uint32_t x, bool border,
                      uint32_t* parent_count, bool* parent_root) {
  node<32> pn, b, a;
  if (!lock_live(t, p, parent, pn)) return t.shfl((uint32_t)fatal_error(p), 0) ? STEP_ERROR : STEP_WALK;
  const int i = pn.is_border() ? -1 : pn.child_slot_of(t, x);
  if (i < 0) {  // merged away, or a root collapsed since the walk
    unlock_node(t, p, parent);
    return STEP_WALK;
  }
  const uint32_t n = pn.count();
  *parent_count = n;
  *parent_root = pn.is_root();
  if (!lock_live(t, p, x, b)) {
    unlock_node(t, p, parent);
    return STEP_ERROR;
  }
  if (b.is_border() != border || b.count() > kMergeAt) {
    unlock_node(t, p, x);
    unlock_node(t, p, parent);
    return b.is_border() != border ? STEP_WALK : STEP_KEPT;
  }
  // Into the left neighbour: the parent's entry i-1 goes, entry i (the
  // separator of x's range) now routes to the neighbour.
  if (i >= 1) {
    const uint32_t left = pn.val_at(t, (uint32_t)i - 1u);
    if (!lock_live(t, p, left, a)) {
      unlock_node(t, p, x);
      unlock_node(t, p, parent);
      return STEP_ERROR;
    }
    if (a.count() + b.count() <= (uint32_t)kMaxEntries) {
      absorb(t, a, b);
      publish_unlock(t, p, a);
      pn.remove_at(t, (uint32_t)i - 1u);
      pn.set_entry(t, (uint32_t)i - 1u, left, 0u);
      publish_unlock(t, p, pn);
      give_up(t, p, b);
      *parent_count = pn.count();
      return STEP_MERGED;
    }
    unlock_node(t, p, left);
  }
  // Else the right neighbour into x: entry i goes, entry i+1 routes to x.
  if ((uint32_t)i + 1u < n) {
    const uint32_t right = pn.val_at(t, (uint32_t)i + 1u);
    if (!lock_live(t, p, right, a)) {
      unlock_node(t, p, x);
      unlock_node(t, p, parent);
      return STEP_ERROR;
    }
    if (a.count() + b.count() <= (uint32_t)kMaxEntries) {
      absorb(t, b, a);
      publish_unlock(t, p, b);
      pn.remove_at(t, (uint32_t)i);
      pn.set_entry(t, (uint32_t)i, x, 0u);
      publish_unlock(t, p, pn);
      give_up(t, p, a);
      *parent_count = pn.count();
      return STEP_MERGED;
    }
    unlock_node(t, p, right);
  }
  unlock_node(t, p, x);
  unlock_node(t, p, parent);
  return STEP_KEPT;
}

// While the layer root is an interior node with one child, the root takes the
// child's entries, kind and range (it keeps its slab and ROOT flag) and the
// child is given up.
MT_DEV void collapse_root(const tile<32>& t, const pool_view& p, uint32_t root) {
  node<32> r, c;
  for (uint32_t k = 0; k < kMaxPath; ++k) {
    if (!lock_live(t, p, root, r)) return;
    if (r.is_border() || r.count() != 1u || !r.is_root()) {
      unlock_node(t, p, root);
      return;
    }
    const uint32_t ch = r.val_at(t, 0u);
    if (!lock_live(t, p, ch, c)) {
      unlock_node(t, p, root);
      return;
    }
    if (c.has_sib()) {  // an only child covers the whole layer
      if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_MERGE));
      unlock_node(t, p, ch);
      unlock_node(t, p, root);
      return;
    }
#pragma unroll
    for (int w = 0; w < node<32>::W; ++w) r.w[w] = c.w[w];
    r.meta = (r.meta & ~(META_COUNT | META_BORDER | META_SIB)) | (c.meta & (META_COUNT | META_BORDER));
    r.ks = c.ks;
    r.high = 0xFFFFFFFFu;
    r.sib = kInvalid;
    publish_unlock(t, p, r);
    give_up(t, p, c);
  }
}

// Merge the border node covering `slice` in the layer rooted at `root`, then
// each ancestor on its path that holds kMergeAt entries or fewer (whether or
// not the level below merged: a sparse parent may be left from an earlier
// call); a root left with one child takes it in.  A stale path is walked
// again and the work resumes at the same height (heights below the root do not
// change in these passes).
MT_DEV void merge_up(const tile<32>& t, const pool_view& p, uint32_t root, uint32_t slice) {
  merge_path mp;
  uint32_t h = 0;  // height of the node to merge next (0: the border node)
  for (uint32_t walk = 0; walk < kMergeWalks; ++walk) {
    if (!walk_path(t, p, root, slice, mp)) return;
    while (true) {
      if (h + 1u >= mp.n) return;  // the node at height h is the root
      const uint32_t j = mp.n - 1u - h;
      uint32_t pc = 0;
      bool proot = false;
      const int r = merge_step(t, p, mp.idx[j - 1u], mp.idx[j], h == 0u, &pc, &proot);
      if (r == STEP_WALK) break;
      if (r == STEP_ERROR) return;
      if (proot) {
        if (pc == 1u) collapse_root(t, p, mp.idx[j - 1u]);
        return;
      }
      if (pc > kMergeAt) return;
      ++h;
    }
  }
}

__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) merge_kernel(tree_view tv, const uint32_t* log,
                                                                              uint32_t cap) {
  tile<32> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  const uint32_t n = min(log[0], cap);
  for (uint32_t r = tile_id; r < n; r += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    merge_up(t, tv.pool, log[2u + 2u * r], log[3u + 2u * r]);
  }
}

// Remove the layer that record `rec` names, then every layer above it that the
// removal leaves without entries (with merges: once the border node that lost
// the LINK entry has been merged upwards and the layer folded into its root).
MT_DEV void remove_layers(const tile<32>& t, const tree_view& tv, const uint32_t* rec, bool merges) {
  const pool_view& p = tv.pool;
  node<32> nd, cn;
  uint32_t walks = 0;
  for (uint32_t depth = rec[0]; depth >= 1u && depth < kLayerRecWords;) {
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
    if (nd.dead()) {  // folded into a neighbour by a merge of this pass since the descent
      unlock_node(t, p, nd.idx);
      if (++walks >= kMergeWalks) return;
      continue;
    }
    const int e = nd.match(t, slice, true);
    if (e < 0 || ks_get(nd.ks, (uint32_t)e) != KS_LINK) {
      unlock_node(t, p, nd.idx);
      return;
    }
    const uint32_t child = nd.val_at(t, (uint32_t)e);
    if (!lock_live(t, p, child, cn)) {
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
    give_up(t, p, cn);
    if (nd.is_root()) {
      if (nd.count() != 0u || nd.has_sib()) return;
    } else {
      if (!merges || nd.count() > kMergeAt) return;
      merge_up(t, p, root, slice);
      if (!nd.template load_verified<kConc>(t, p, root)) return;
      if (!nd.is_border() || nd.count() != 0u || nd.has_sib()) return;
    }
    --depth;
  }
}

__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) remove_layers_kernel(tree_view tv,
                                                                                      const uint32_t* log,
                                                                                      uint32_t cap, bool merges) {
  tile<32> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  const uint32_t n = min(log[0], cap);
  for (uint32_t r = tile_id; r < n; r += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    remove_layers(t, tv, log + 2u + (size_t)kLayerRecWords * r, merges);
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
  if (layers)
    remove_layers_kernel<<<std::max(1, t->sms * 4), kBlock, 0, s>>>(t->tv, t->layer_log, kLayerCap, merges);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

}  // namespace mtb
