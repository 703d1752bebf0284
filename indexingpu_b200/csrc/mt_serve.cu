// Serving: a device-resident request loop with continuous admission (mt_serve).
//
// Requests (1..n ops of any kind) arrive over time.  The host side publishes
// each admitted request as work items of at most `chunk_ops` ops into a
// descriptor ring in pinned, device-mapped host memory and bumps a published
// counter.  A persistent kernel (one warp per work item at a time) claims
// items with a compare-and-swap on a device counter, serves their ops with the
// mixed-request code of the batch kernels, and when the last item of a request
// finishes writes the request's completion flag back to host memory.  Work of
// requests that arrive while others run is admitted at once and overlaps with
// them on the device; nothing waits for a batch to fill.
//
// Safety and reclamation: every launch of the server kernel ends by itself
// after `epoch_us` of device time (or at once when the host raises stop), so no
// wait is unbounded; the host relaunches it back to back, with the reclaim pass
// in between returning the slabs retired during the previous launch.
// Admission: a request is published only while the slabs the admitted
// requests may consume (two per insert or update, at most) keep the pool under
// `memory_budget` of its slabs.
//
// The same entry point runs the plain form for comparison: one synchronous
// mt_mixed_batch call per request, in arrival order.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "mt_internal.cuh"

namespace mtb {

struct __align__(16) serve_item {   // one work item: ops [first, first + count) of request `req`
  uint32_t req;
  uint32_t first;
  uint32_t count;
  uint32_t items;     // work items of the request
};

// Device-side control words of one serving run.  Items are claimed by
// fetch-and-add tickets, taken before the item is published: a warp holds one
// ticket and waits for the host to publish it, so a claim costs one atomic and
// idle warps only read.  The waiting warps read one of kReplicas copies of
// the published count (each on its own 128-byte line, so that thousands of
// pollers spread over L2 slices instead of queueing on one); only the warp
// holding the first unpublished ticket (the head) reads the host's counter and
// stop flag and updates the copies.  A ticket still unpublished when a launch
// ends stays in the warp's slot of `held`; every launch has the same grid, so
// the same warp of the next launch resumes it and every ticket is served
// exactly once.
constexpr int kReplicas = 16;
struct __align__(128) pub_replica {
  unsigned long long pub;  // published items (monotonic)
  uint32_t stop;           // host asked the loop to end
  uint32_t pad[29];
};
struct __align__(128) server_ctl {
  unsigned long long next;  // tickets taken so far
  uint32_t pad[30];
  pub_replica rep[kReplicas];
};

struct server_view {
  const serve_item* ring;               // mapped host memory
  const unsigned long long* published;  // mapped host: items published so far
  const uint32_t* stop;                 // mapped host: 1 = leave now
  server_ctl* ctl;                      // device
  unsigned long long* held;             // device: per warp of the grid, a ticket carried over (~0: none)
  uint32_t* finished;                   // device: finished items per request
  uint32_t* done;                       // mapped host: per-request completion flags
  uint32_t ring_cap;
  const uint32_t* order;                // device: op indexes, every request's ops grouped by kind
  batch_args ops;                       // op arrays of all requests
};

MT_DEV unsigned long long ld_acquire_sys_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
// A ring entry lives in host memory: read it at system scope.
MT_DEV serve_item ld_item(const serve_item* p) {
  serve_item it;
  asm volatile("ld.relaxed.sys.global.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(it.req), "=r"(it.first), "=r"(it.count), "=r"(it.items) : "l"(p) : "memory");
  return it;
}
MT_DEV unsigned long long ld_acquire_gpu_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
MT_DEV void atom_max_release_gpu_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.max.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
MT_DEV uint32_t atom_add_acq_rel_gpu_u32(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
MT_DEV uint32_t ld_sys_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
MT_DEV unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

MT_DEV void st_relaxed_sys_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.sys.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Head of the ticket queue: read the host's published counter and stop flag
// and spread them to every replica.  Returns the freshest published count.
MT_DEV unsigned long long head_refresh(const server_view& sv, unsigned long long known) {
  server_ctl* ctl = sv.ctl;
  const unsigned long long hp = ld_acquire_sys_u64(sv.published);
  if (hp > known) {
    // The release passes the ring entries seen through hp on to every warp
    // that reads the new count with acquire.
#pragma unroll 1
    for (int i = 0; i < kReplicas; ++i) atom_max_release_gpu_u64(&ctl->rep[i].pub, hp);
    return hp;
  }
  if (ld_sys_u32(sv.stop) != 0u) {
#pragma unroll 1
    for (int i = 0; i < kReplicas; ++i) *(volatile uint32_t*)&ctl->rep[i].stop = 1u;
  }
  return known;
}

template <int T>
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) server_kernel(tree_view tv, server_view sv,
                                                                              unsigned long long budget_ns) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long deadline = global_ns() + budget_ns;  // used by lane 0 only
  tile<T> t;
  slab_cache<T> cache;
  cache.init(tv.pool, (blockIdx.x * blockDim.x + threadIdx.x) / T);
  tile<32> tw;
  slab_cache<32> wcache;
  if (T < 32) wcache.init(tv.pool, (blockIdx.x * blockDim.x + threadIdx.x) / 32u);
  constexpr uint32_t tiles_per_warp = 32u / T;
  const uint32_t tile_in_warp = lane / T;
  server_ctl* ctl = sv.ctl;
  pub_replica* rep = &ctl->rep[blockIdx.x % kReplicas];
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  unsigned long long carried = (lane == 0) ? sv.held[wid] : ~0ull;  // leader only
  unsigned long long keep = ~0ull;                                   // leader: ticket to carry on
  while (true) {
    // Warp leader: hold a ticket and wait (bounded by the launch's deadline)
    // until the host publishes it.
    unsigned long long c = ~0ull;
    uint32_t leave = 0;
    if (lane == 0) {
      c = (carried != ~0ull) ? carried : atomicAdd(&ctl->next, 1ull);
      carried = ~0ull;
      while (true) {
        unsigned long long pubc = ld_acquire_gpu_u64(&rep->pub);
        if (c < pubc) break;
        if (c == pubc) {  // head of the queue: ask the host
          pubc = head_refresh(sv, pubc);
          if (c < pubc) break;
        }
        if (*(volatile uint32_t*)&rep->stop != 0u || global_ns() > deadline) {
          keep = c;  // the next launch resumes it
          c = ~0ull;
          leave = 1u;
          break;
        }
        __nanosleep(c == pubc ? 100 : 400);
      }
    }
    c = __shfl_sync(0xFFFFFFFFu, c, 0);
    leave = __shfl_sync(0xFFFFFFFFu, leave, 0);
    if (leave) break;
    const serve_item it = ld_item(sv.ring + (c % sv.ring_cap));
    // The item's ops, through the kind-grouped order: the tiles of a warp
    // mostly serve ops of one kind side by side (one code path, no
    // divergence between find and write paths).
    batch_args a = sv.ops;
    a.index = sv.order + it.first;
    a.n_dev = nullptr;
    a.n_back_dev = nullptr;
    a.n = it.count;
    // Items are cut from each request's ops in kind order (finds first): an
    // item that starts with a write holds writes only, and the whole warp
    // serves it as one 32-lane tile, the width writes run best at (as the
    // write classes of a mixed batch); finds keep the narrow tiles.
    uint32_t k0 = 0;
    if (T < 32 && lane == 0 && it.count > 0u) k0 = a.types[a.index[0]];
    if (T < 32 && __shfl_sync(0xFFFFFFFFu, k0, 0) != (uint32_t)MT_REQ_FIND) {
      serve_requests<32, OP_MIXED, true>(tw, tv, wcache, a, 0u, 1u);
    } else {
      serve_requests<T, OP_MIXED, true>(t, tv, cache, a, tile_in_warp, tiles_per_warp);
    }
    __syncwarp();
    if (lane == 0) {
      // acq_rel: the last item of a request has seen every write of the
      // others, all in device memory, before it raises the request's flag
      // (the host reads results only through later copies or calls).
      const uint32_t f = atom_add_acq_rel_gpu_u32(sv.finished + it.req, 1u) + 1u;
      if (f == it.items) {
        // The counter starts again at 0 for the next request of this slot
        // (mt_server_* reuses slots); the system-scope fence makes every
        // result of the request visible to the host's copies before the flag.
        atomicExch(sv.finished + it.req, 0u);
        __threadfence_system();
        st_relaxed_sys_u32(sv.done + it.req, 1u);
      } else if (f > it.items) {
        record_error(tv.pool, ERR_CORRUPT, MT_AT(SRC_SERVE));  // an item served twice
      }
    }
    // Warp-uniform: lane 0 reads the clock and decides for the whole warp
    // (every lane's own reading could split the warp).
    if (__shfl_sync(0xFFFFFFFFu, (lane == 0 && global_ns() > deadline) ? 1u : 0u, 0)) break;
  }
  if (lane == 0) sv.held[wid] = keep;
  cache.release(t, tv.pool);
  if (T < 32) wcache.release(tw, tv.pool);
}

// Slabs handed out and not yet back on a free stack (in use + limbo), written
// to mapped host memory after each reclaim pass for the admission estimate.
__global__ void pool_usage_kernel(pool_view p, unsigned long long* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long held = 0;
  for (uint32_t s = 0; s < p.num_shards; ++s) {
    const int bump = *(volatile int*)p.bump(s);
    const int top = *(volatile int*)p.top(s);
    const unsigned long long handed = (unsigned long long)min(max(bump, 0), (int)p.shard_slabs);
    held += handed - min(handed, (unsigned long long)max(top, 0));
  }
  *(volatile unsigned long long*)out = held;
}

}  // namespace mtb

using namespace mtb;

namespace {

using clk = std::chrono::steady_clock;

uint64_t now_ns(clk::time_point t0) {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count();
}

template <int T>
int server_blocks(mt_masstree* t) {
  int bps = host_max_blocks_per_sm((const void*)server_kernel<T>, kBlock, 0);
  if (t->blocks_per_sm > 0) bps = std::min<int>(bps, (int)t->blocks_per_sm);
  return std::max(bps, 1) * t->sms;
}

int server_blocks_tile(mt_masstree* t) {
  switch (t->tile_size) {
    case 4: return server_blocks<4>(t);
    case 8: return server_blocks<8>(t);
    case 16: return server_blocks<16>(t);
    default: return server_blocks<32>(t);
  }
}

// Every launch of one run has the same grid (the per-warp ticket slots rely
// on it).
int launch_server_tile(mt_masstree* t, int blocks, const server_view& sv, unsigned long long budget_ns,
                       cudaStream_t s) {
  switch (t->tile_size) {
    case 4: server_kernel<4><<<blocks, kBlock, 0, s>>>(t->tv, sv, budget_ns); break;
    case 8: server_kernel<8><<<blocks, kBlock, 0, s>>>(t->tv, sv, budget_ns); break;
    case 16: server_kernel<16><<<blocks, kBlock, 0, s>>>(t->tv, sv, budget_ns); break;
    default: server_kernel<32><<<blocks, kBlock, 0, s>>>(t->tv, sv, budget_ns); break;
  }
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

// Pinned, device-mapped host allocation.
template <typename X>
X* mapped_alloc(size_t n, X** dev) {
  void* h = nullptr;
  if (cudaHostAlloc(&h, std::max<size_t>(n, 1) * sizeof(X), cudaHostAllocMapped) != cudaSuccess) return nullptr;
  std::memset(h, 0, std::max<size_t>(n, 1) * sizeof(X));
  void* d = nullptr;
  if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
    cudaFreeHost(h);
    return nullptr;
  }
  *dev = static_cast<X*>(d);
  return static_cast<X*>(h);
}

}  // namespace

namespace {
int serve_online(mt_masstree* t, const mt_serve_plan* plan, uint64_t* latency_ns, mt_serve_stats* stats);
}  // namespace

extern "C" int mt_serve(mt_masstree* t, const mt_serve_plan* plan, uint64_t* latency_ns, mt_serve_stats* stats) {
  if (!t || !plan || !latency_ns || plan->num_requests == 0 || !plan->request_first_op || !plan->request_num_ops ||
      !plan->arrival_ns || !plan->types || !plan->keys || !plan->values || !plan->value_lengths ||
      plan->max_key_length == 0 || plan->max_value_length == 0 ||
      (plan->mode != MT_SERVE_SERVED && plan->mode != MT_SERVE_PLAIN && plan->mode != MT_SERVE_ONLINE))
    return MT_ERR_INVALID_ARG;
  if (plan->mode == MT_SERVE_ONLINE) return serve_online(t, plan, latency_ns, stats);
  const uint32_t nreq = plan->num_requests;
  uint64_t total_ops = 0;
  for (uint32_t r = 0; r < nreq; ++r) {
    // Requests are given in arrival order.
    if (r > 0 && plan->arrival_ns[r] < plan->arrival_ns[r - 1]) return MT_ERR_INVALID_ARG;
    total_ops = std::max<uint64_t>(total_ops, (uint64_t)plan->request_first_op[r] + plan->request_num_ops[r]);
  }
  if (total_ops > 0xFFFFFFFFull) return MT_ERR_INVALID_ARG;
  {
    // Every op belongs to at most one request.
    std::vector<uint8_t> owned(std::max<uint64_t>(total_ops, 1), 0);
    for (uint32_t r = 0; r < nreq; ++r)
      for (uint32_t o = plan->request_first_op[r]; o < plan->request_first_op[r] + plan->request_num_ops[r]; ++o) {
        if (owned[o]) return MT_ERR_INVALID_ARG;
        owned[o] = 1;
      }
  }
  // Work-item size: fixed, or (chunk_ops == 0) chosen per request from the
  // backlog (ops admitted and not complete): one op per item (a warp each,
  // lowest latency) while the backlog is below an eighth of the grid's warps, then
  // one, two, four or eight ops per tile of a warp as it grows (fewer items
  // per op: one-op items cap the loop at about a sixth of its peak).
  const uint32_t tiles_per_warp = 32u / t->tile_size;
  const bool auto_chunk = plan->chunk_ops == 0;
  const uint32_t fixed_chunk = std::max<uint32_t>(1u, std::min<uint32_t>(plan->chunk_ops, 4096u));
  const uint32_t min_chunk = auto_chunk ? 1u : fixed_chunk;
  const double budget = plan->memory_budget > 0.f ? plan->memory_budget : 0.9;
  mt_stats_t st{};
  int rc = mt_stats(t, &st);
  if (rc) return rc;
  const double slab_budget = budget * (double)st.total_slabs;
  double slabs_in_use = (double)st.used_slabs + (double)st.limbo_slabs;
  std::vector<uint8_t> h_types;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return MT_ERR_CUDA;
  uint64_t admitted = 0, rejected_waits = 0;
  std::vector<uint64_t> arrival(nreq), completion(nreq, 0);
  // Per-request slab demand estimate: per insert or update, a suffix chain of
  // the maximum lengths plus one slab for a node split.
  std::vector<uint32_t> demand(nreq, 0);
  const uint32_t per_write = 1u + suf_nodes(plan->max_key_length, plan->max_value_length);
  {
    h_types.resize(std::max<uint64_t>(total_ops, 1));
    if (total_ops && cudaMemcpy(h_types.data(), plan->types, total_ops, cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaStreamDestroy(s);
      return MT_ERR_CUDA;
    }
    for (uint32_t r = 0; r < nreq; ++r) {
      uint32_t d = 0;
      for (uint32_t o = 0; o < plan->request_num_ops[r]; ++o) {
        const uint8_t k = h_types[plan->request_first_op[r] + o];
        d += (k == MT_REQ_INSERT || k == MT_REQ_UPDATE) ? per_write : 0u;
      }
      demand[r] = d;
    }
  }
  batch_args ops{};
  ops.types = plan->types;
  ops.keys = plan->keys;
  ops.key_lengths = plan->key_lengths;
  ops.values = plan->values;
  ops.value_lengths_in = plan->value_lengths;
  ops.value_lengths_out = plan->value_lengths;
  ops.results = plan->results;
  ops.max_key_length = plan->max_key_length;
  ops.max_value_length = plan->max_value_length;

  clk::time_point t0;  // time 0 of the arrival schedule, taken once set-up is done
  if (plan->mode == MT_SERVE_PLAIN) {
    // One synchronous mixed_batch call per request, in arrival order.
    t0 = clk::now();
    for (uint32_t r = 0; r < nreq; ++r) {
      while (now_ns(t0) < plan->arrival_ns[r]) {
      }
      arrival[r] = plan->arrival_ns[r];
      const uint32_t f = plan->request_first_op[r];
      rc = mt_mixed_batch(t, plan->types + f, plan->keys + (size_t)f * plan->max_key_length, plan->max_key_length,
                          plan->key_lengths ? plan->key_lengths + f : nullptr,
                          plan->values + (size_t)f * plan->max_value_length, plan->max_value_length,
                          plan->value_lengths + f, plan->results ? plan->results + f : nullptr,
                          plan->request_num_ops[r], 0u, s);
      if (rc) break;
      if (cudaStreamSynchronize(s) != cudaSuccess) { rc = MT_ERR_CUDA; break; }
      completion[r] = now_ns(t0);
      ++admitted;
    }
  } else {
    // Device-resident loop.
    uint64_t total_items = 0;  // ring capacity: every request cut at the smallest item size
    for (uint32_t r = 0; r < nreq; ++r)
      total_items += std::max<uint32_t>(1u, (plan->request_num_ops[r] + min_chunk - 1) / min_chunk);
    serve_item* d_ring = nullptr;
    unsigned long long* d_pub = nullptr;
    uint32_t *d_stop = nullptr, *d_done = nullptr, *d_finished = nullptr;
    unsigned long long* d_usage = nullptr;
    unsigned long long* d_held = nullptr;
    uint32_t* d_order = nullptr;
    server_ctl* d_ctl = nullptr;
    const int blocks = server_blocks_tile(t);
    const size_t nwarps = (size_t)blocks * (kBlock / 32);
    serve_item* ring = mapped_alloc<serve_item>(total_items, &d_ring);
    unsigned long long* pub = mapped_alloc<unsigned long long>(1, &d_pub);
    uint32_t* stop = mapped_alloc<uint32_t>(1, &d_stop);
    uint32_t* done = mapped_alloc<uint32_t>(nreq, &d_done);
    unsigned long long* usage = mapped_alloc<unsigned long long>(1, &d_usage);
    bool ok = ring && pub && stop && done && usage;
    if (ok) ok = cudaMalloc(&d_finished, (size_t)nreq * sizeof(uint32_t)) == cudaSuccess &&
                 cudaMalloc(&d_ctl, sizeof(server_ctl)) == cudaSuccess &&
                 cudaMalloc(&d_held, nwarps * sizeof(unsigned long long)) == cudaSuccess &&
                 cudaMemset(d_held, 0xFF, nwarps * sizeof(unsigned long long)) == cudaSuccess &&
                 cudaMemset(d_finished, 0, (size_t)nreq * sizeof(uint32_t)) == cudaSuccess &&
                 cudaMemset(d_ctl, 0, sizeof(server_ctl)) == cudaSuccess;
    if (ok) {
      // Every request's ops in the order finds, inserts, updates and erases
      // (a request's ops have no order among each other, as in one mixed
      // batch), so that items cut from it are mostly of one kind.
      std::vector<uint32_t> order(std::max<uint64_t>(total_ops, 1));
      for (uint32_t r = 0; r < nreq; ++r) {
        const uint32_t f = plan->request_first_op[r], no = plan->request_num_ops[r];
        uint32_t pos = f;
        for (uint8_t kind : {(uint8_t)MT_REQ_FIND, (uint8_t)MT_REQ_INSERT, (uint8_t)MT_REQ_UPDATE,
                             (uint8_t)MT_REQ_ERASE})
          for (uint32_t o = f; o < f + no; ++o)
            if (h_types[o] == kind) order[pos++] = o;
        for (uint32_t o = f; o < f + no; ++o)  // unknown kinds: served (and reported) last
          if (h_types[o] > MT_REQ_UPDATE) order[pos++] = o;
      }
      ok = cudaMalloc(&d_order, order.size() * sizeof(uint32_t)) == cudaSuccess &&
           cudaMemcpy(d_order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) ==
               cudaSuccess;
    }
    if (usage) *usage = (unsigned long long)slabs_in_use;
    server_view sv{};
    sv.ring = d_ring;
    sv.published = d_pub;
    sv.stop = d_stop;
    sv.ctl = d_ctl;
    sv.held = d_held;
    sv.finished = d_finished;
    sv.done = d_done;
    sv.ring_cap = (uint32_t)std::min<uint64_t>(total_items, 0xFFFFFFFFull);
    sv.order = d_order;
    sv.ops = ops;
    const unsigned long long epoch_ns = (unsigned long long)(plan->epoch_us ? plan->epoch_us : 20000u) * 1000ull;
    if (ok) {
      // One launch with no time budget before the clock starts: it loads the
      // kernels and leaves every warp holding its first ticket.
      ok = host_launch_reclaim(t, s) == MT_OK && launch_server_tile(t, blocks, sv, 0ull, s) == MT_OK;
      pool_usage_kernel<<<1, 32, 0, s>>>(t->tv.pool, d_usage);
      ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    }
    if (ok) {
      t0 = clk::now();
      std::atomic<uint32_t> completed{0};
      std::atomic<uint64_t> completed_demand{0};
      std::atomic<uint64_t> completed_ops{0};
      uint64_t admitted_ops = 0;
      const uint64_t total_tiles = nwarps * tiles_per_warp;
      uint32_t waiting_for = ~0u;
      std::atomic<bool> poll_stop{false};
      uint64_t admitted_demand = 0;
      std::vector<uint64_t> enq_completed;  // completed_demand when each epoch was enqueued
      // Completion poller: watches only the requests admitted and not yet
      // complete, so a pass costs O(requests in flight).
      std::atomic<uint32_t> admitted_count{0};
      std::thread poller([&] {
        std::vector<uint32_t> pending;
        uint32_t known = 0;
        while (completed.load(std::memory_order_relaxed) < nreq && !poll_stop.load(std::memory_order_relaxed)) {
          const uint32_t adm = admitted_count.load(std::memory_order_acquire);
          while (known < adm) pending.push_back(known++);
          bool progress = false;
          for (size_t i = 0; i < pending.size();) {
            const uint32_t q = pending[i];
            if (__atomic_load_n(&done[q], __ATOMIC_ACQUIRE)) {
              completion[q] = now_ns(t0);
              completed_demand.fetch_add(demand[q]);
              completed_ops.fetch_add(plan->request_num_ops[q]);
              completed.fetch_add(1);
              pending[i] = pending.back();
              pending.pop_back();
              progress = true;
            } else {
              ++i;
            }
          }
          if (!progress && pending.empty()) std::this_thread::yield();
        }
      });
      // Epoch launcher: keep two launches queued.
      std::vector<cudaEvent_t> evs;
      auto enqueue_epoch = [&]() -> int {
        int r2 = host_launch_reclaim(t, s);
        if (r2) return r2;
        pool_usage_kernel<<<1, 32, 0, s>>>(t->tv.pool, d_usage);
        r2 = launch_server_tile(t, blocks, sv, epoch_ns, s);
        if (r2) return r2;
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MT_ERR_CUDA;
        cudaEventRecord(e, s);
        evs.push_back(e);
        enq_completed.push_back(completed_demand.load());
        return MT_OK;
      };
      size_t ev_done = 0;
      rc = enqueue_epoch();
      if (!rc) rc = enqueue_epoch();
      uint64_t published = 0;
      uint32_t r = 0;
      while (!rc && (r < nreq || completed.load() < nreq)) {
        // Publish every request whose arrival time has come, if memory allows.
        const uint64_t now = now_ns(t0);
        while (r < nreq && plan->arrival_ns[r] <= now) {
          if (slabs_in_use + demand[r] > slab_budget) {
            // Admission waits for memory (slabs come back between launches).
            if (waiting_for != r) { ++rejected_waits; waiting_for = r; }
            break;
          }
          arrival[r] = plan->arrival_ns[r];
          uint32_t chunk = fixed_chunk;
          if (auto_chunk) {
            const uint64_t backlog = admitted_ops - std::min(admitted_ops, completed_ops.load());
            const uint64_t per_tile = backlog / total_tiles;
            chunk = backlog < nwarps / 8 ? 1u
                                         : tiles_per_warp * (per_tile < 1 ? 1u : per_tile < 2 ? 2u : per_tile < 4 ? 4u : 8u);
          }
          const uint32_t nops = plan->request_num_ops[r];
          const uint32_t n_items = std::max<uint32_t>(1u, (nops + chunk - 1) / chunk);
          admitted_ops += nops;
          uint32_t f = plan->request_first_op[r];
          uint32_t left = nops;
          for (uint32_t k = 0; k < n_items; ++k) {
            const uint32_t c = std::min(left, chunk);
            ring[published % sv.ring_cap] = serve_item{r, f, c, n_items};
            ++published;
            f += c;
            left -= c;
          }
          __atomic_store_n(pub, (unsigned long long)published, __ATOMIC_RELEASE);
          slabs_in_use += demand[r];
          admitted_demand += demand[r];
          ++admitted;
          ++r;
          admitted_count.store(r, std::memory_order_release);
        }
        // Keep the device loop running.
        while (ev_done < evs.size() && cudaEventQuery(evs[ev_done]) == cudaSuccess) {
          ++ev_done;
          if (r < nreq || completed.load() < nreq) rc = enqueue_epoch();
          // Retired slabs came back with the reclaim pass before that launch.
          // Restart the estimate from the pool count taken then, plus the
          // demand of every request not complete when that epoch was enqueued
          // (requests complete by then are fully in the count): an upper bound.
          slabs_in_use = (double)__atomic_load_n(usage, __ATOMIC_ACQUIRE) +
                         (double)(admitted_demand - std::min(admitted_demand, enq_completed[ev_done - 1]));
        }
        if (now_ns(t0) > plan->arrival_ns[nreq - 1] + 60ull * 1000000000ull) {
          // Bounded run: a request that never fitted the memory budget, or
          // work that never completed.
          rc = r < nreq ? MT_ERR_OOM : MT_ERR_LOCK_TIMEOUT;
          break;
        }
      }
      __atomic_store_n(stop, 1u, __ATOMIC_RELEASE);
      cudaStreamSynchronize(s);
      poll_stop.store(true);
      poller.join();
      for (auto e : evs) cudaEventDestroy(e);
    } else {
      rc = MT_ERR_OOM;
    }
    if (ring) cudaFreeHost(ring);
    if (pub) cudaFreeHost(pub);
    if (stop) cudaFreeHost(stop);
    if (done) cudaFreeHost(done);
    if (usage) cudaFreeHost(usage);
    if (d_finished) cudaFree(d_finished);
    if (d_ctl) cudaFree(d_ctl);
    if (d_held) cudaFree(d_held);
    if (d_order) cudaFree(d_order);
  }
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  uint64_t ops_done = 0, end = 0;
  for (uint32_t r = 0; r < nreq; ++r) {
    latency_ns[r] = completion[r] ? completion[r] - arrival[r] : 0ull;
    if (completion[r]) ops_done += plan->request_num_ops[r];
    end = std::max<uint64_t>(end, completion[r]);
  }
  if (stats) {
    stats->wall_ns = end;
    stats->requests_done = admitted;
    stats->ops_done = ops_done;
    stats->admission_waits = rejected_waits;
    for (uint64_t& x : stats->stage_ns) x = 0;
  }
  if (!rc) rc = mt_sync(t, nullptr);
  return rc;
}

// ---- online serving (mt_server_*) ------------------------------------------------------
//
// The device loop above, fed while it runs.  Clients call mt_server_submit
// from any host thread; the server's own host thread (the pump) moves each
// request through: queued -> admitted (staging space, a request slot and the
// memory budget allow) -> uploading -> published (work items on the ring) ->
// done.  Per pump round, the requests admitted together are copied (CPU) into
// a pinned host staging ring and go to the device with ONE copy per field; the
// device loop writes find values, value lengths and write results straight
// into mapped host memory, and when the device raises a request's completion
// flag the pump copies its results into the client's buffers and marks the
// ticket done.  Staging is a ring of max_ops_in_flight ops, filled and freed
// in admission order; request slots are ticket % max_requests_in_flight.

namespace {

enum : uint32_t { SRV_UPLOADING = 0, SRV_PUBLISHED = 1, SRV_DONE = 2 };

struct srv_request {
  uint64_t ticket = 0;
  const uint8_t* types = nullptr;
  const uint32_t* keys = nullptr;
  const uint32_t* klens = nullptr;
  uint32_t* vals = nullptr;
  uint32_t* vlens = nullptr;
  bool* results = nullptr;
  uint32_t n = 0;
  uint64_t submit_ns = 0;
  uint64_t admit_ns = 0, publish_ns = 0, done_ns = 0;  // stage times (mt_server_stats)
  uint32_t off = 0;        // staging offset of the request's ops
  uint64_t alloc_end = 0;  // staging head after its allocation
  uint32_t demand = 0;     // slab demand estimate
  uint32_t stage = SRV_UPLOADING;
};

struct srv_round {  // requests admitted in one pump round, uploaded together
  cudaEvent_t ev = nullptr;
  std::vector<uint32_t> slots;
};

// A few host threads that help the pump copy requests in and results out
// (one host core moving about 100 bytes per op in and out caps the server
// far below the device loop).  run(n, f) calls f(0..n-1) on the pool and the
// caller and returns when all calls have ended and no worker is in the loop.
struct copy_pool {
  std::vector<std::thread> th;
  std::mutex mu;
  std::condition_variable cv;
  std::function<void(size_t)> fn;
  size_t n = 0;
  uint64_t gen = 0;
  bool stop = false;
  std::atomic<size_t> next{0}, finished{0};
  std::atomic<int> active{0};
  std::atomic<uint64_t> gen_seen{0};  // gen, readable without the lock (polling workers)
  std::atomic<bool> stop_seen{false};

  void start(int workers) {
    for (int k = 0; k < workers; ++k) th.emplace_back([this] { loop(); });
  }
  void loop() {
    uint64_t seen = 0;
    while (true) {
      // Poll for new work for a while (a sleeping worker takes tens of
      // microseconds to wake), then sleep until notified.
      for (int spin = 0; spin < 20000 && gen_seen.load(std::memory_order_acquire) == seen &&
                         !stop_seen.load(std::memory_order_acquire);
           ++spin)
        std::this_thread::yield();
      std::function<void(size_t)> f;
      size_t cnt = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || gen != seen; });
        if (stop) return;
        seen = gen;
        f = fn;
        cnt = n;
        active.fetch_add(1);
      }
      for (size_t k; (k = next.fetch_add(1)) < cnt;) {
        f(k);
        finished.fetch_add(1);
      }
      active.fetch_sub(1);
    }
  }
  void run(size_t cnt, const std::function<void(size_t)>& f) {
    if (th.empty() || cnt < 2) {
      for (size_t k = 0; k < cnt; ++k) f(k);
      return;
    }
    {
      std::lock_guard<std::mutex> g(mu);
      fn = f;
      n = cnt;
      next = 0;
      finished = 0;
      ++gen;
      gen_seen.store(gen, std::memory_order_release);
    }
    cv.notify_all();
    for (size_t k; (k = next.fetch_add(1)) < cnt;) {
      f(k);
      finished.fetch_add(1);
    }
    while (finished.load() < cnt || active.load() != 0) std::this_thread::yield();
  }
  ~copy_pool() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
      stop_seen.store(true, std::memory_order_release);
    }
    cv.notify_all();
    for (auto& x : th) x.join();
  }
};

constexpr uint64_t kPoolMinOps = 4096;     // rounds this large are copied by the pool
constexpr int kUpStreams = 3;              // upload streams of the online server
constexpr uint64_t kRoundMaxOps = 1u << 17;  // a round admits at most this many ops (then uploads)

}  // namespace

struct mt_server {
  mt_masstree* tree = nullptr;
  mt_server_config cfg{};
  uint32_t C = 0, R = 0;
  uint32_t L = 0;  // completion records: ticket % L (at least 65,536 tickets back, whatever R)
  // Device staging of the inputs, and its pinned host mirror.
  void* dmem = nullptr;
  uint8_t* d_types = nullptr;
  uint32_t *d_keys = nullptr, *d_klens = nullptr, *d_vals = nullptr, *d_vlens = nullptr, *d_order = nullptr;
  void* hmem = nullptr;
  uint8_t* h_types = nullptr;
  uint32_t *h_keys = nullptr, *h_klens = nullptr, *h_vals = nullptr, *h_vlens = nullptr, *h_order = nullptr;
  // Outputs, written by the device into mapped host memory.
  uint32_t *m_vals = nullptr, *m_vals_d = nullptr, *m_vlens = nullptr, *m_vlens_d = nullptr;
  bool *m_results = nullptr, *m_results_d = nullptr;
  serve_item *ring = nullptr, *d_ring = nullptr;
  unsigned long long *pub = nullptr, *d_pub = nullptr;
  uint32_t *stop = nullptr, *d_stop = nullptr, *done = nullptr, *d_done = nullptr;
  unsigned long long *usage = nullptr, *d_usage = nullptr;
  uint32_t* d_finished = nullptr;
  server_ctl* d_ctl = nullptr;
  unsigned long long* d_held = nullptr;
  server_view sv{};
  int blocks = 0;
  size_t nwarps = 0;
  cudaStream_t s_work = nullptr;
  cudaStream_t s_up[kUpStreams] = {};    // uploads (pump only)
  cudaEvent_t up_join[kUpStreams] = {};  // joins the upload streams into s_up[0]
  std::vector<cudaEvent_t> ev_pool;  // pump only
  std::unique_ptr<std::atomic<uint64_t>[]> rec_ticket;
  std::unique_ptr<std::atomic<uint32_t>[]> rec_done;
  std::unique_ptr<std::atomic<uint64_t>[]> rec_latency;
  std::vector<srv_request> slots;  // pump thread only
  copy_pool pool;                  // helps the pump copy (pump thread only)
  std::mutex mu;
  std::deque<srv_request> queued;  // under mu
  std::atomic<uint64_t> next_ticket{0};
  std::thread pump;
  std::atomic<bool> draining{false};  // stop asked: serve what is queued, then end
  std::atomic<bool> quit{false};      // end now (the drain ran out of time)
  std::atomic<bool> exited{false};    // the pump has ended
  std::atomic<int> status{MT_OK};
  clk::time_point t0;
  // Stage sums of completed requests (written by the pump, read by mt_server_stats).
  std::atomic<uint64_t> st_requests{0}, st_ops{0}, st_queued{0}, st_upload{0}, st_device{0}, st_deliver{0},
      st_max{0};
};

namespace {

void server_free(mt_server* S) {
  if (S->s_work) cudaStreamSynchronize(S->s_work);
  for (cudaStream_t st : S->s_up)
    if (st) cudaStreamSynchronize(st);
  for (cudaEvent_t e : S->up_join)
    if (e) cudaEventDestroy(e);
  for (auto e : S->ev_pool) cudaEventDestroy(e);
  if (S->dmem) cudaFree(S->dmem);
  for (void* h : {S->hmem, (void*)S->m_vals, (void*)S->m_vlens, (void*)S->m_results, (void*)S->ring,
                  (void*)S->pub, (void*)S->stop, (void*)S->done, (void*)S->usage})
    if (h) cudaFreeHost(h);
  if (S->d_finished) cudaFree(S->d_finished);
  if (S->d_ctl) cudaFree(S->d_ctl);
  if (S->d_held) cudaFree(S->d_held);
  if (S->s_work) cudaStreamDestroy(S->s_work);
  for (cudaStream_t st : S->s_up)
    if (st) cudaStreamDestroy(st);
  delete S;
}

// Copy request r's inputs into the host staging at r.off and file its ops in
// kind order (finds, inserts, updates, erases: items cut from a request are
// then mostly of one kind, as in mt_serve).
void server_stage(mt_server* S, const srv_request& r) {
  const uint32_t K = S->cfg.max_key_length, V = S->cfg.max_value_length, off = r.off, n = r.n;
  std::memcpy(S->h_types + off, r.types, n);
  std::memcpy(S->h_keys + (size_t)off * K, r.keys, (size_t)n * K * 4u);
  if (r.klens) std::memcpy(S->h_klens + off, r.klens, (size_t)n * 4u);
  else std::fill(S->h_klens + off, S->h_klens + off + n, K);
  std::memcpy(S->h_vals + (size_t)off * V, r.vals, (size_t)n * V * 4u);
  std::memcpy(S->h_vlens + off, r.vlens, (size_t)n * 4u);
  // Outputs start as the inputs: an op the device skips (invalid lengths,
  // reported as MT_ERR_INVALID_ARG) hands its buffers back unchanged.
  std::memcpy(S->m_vlens + off, r.vlens, (size_t)n * 4u);
  if (r.results) std::memcpy(S->m_results + off, r.results, n);
  uint32_t cnt[5] = {0, 0, 0, 0, 0};  // per kind rank: find, insert, update, erase, other
  auto rank = [](uint8_t k) -> int {
    return k == MT_REQ_FIND ? 0 : k == MT_REQ_INSERT ? 1 : k == MT_REQ_UPDATE ? 2 : k == MT_REQ_ERASE ? 3 : 4;
  };
  for (uint32_t o = 0; o < n; ++o) ++cnt[rank(r.types[o])];
  uint32_t start[5];
  uint32_t acc = off;
  for (int k = 0; k < 5; ++k) {
    start[k] = acc;
    acc += cnt[k];
  }
  for (uint32_t o = 0; o < n; ++o) S->h_order[start[rank(r.types[o])]++] = off + o;
}

// Upload staging ops [lo, hi) (one contiguous run): the six fields' copies
// spread over the upload streams, so that the copy engines take them side by
// side (a small copy costs microseconds of set-up; six in a row on one stream
// were most of a small request's upload time).
int server_upload_range(mt_server* S, uint32_t lo, uint32_t hi) {
  if (hi <= lo) return MT_OK;
  const uint32_t K = S->cfg.max_key_length, V = S->cfg.max_value_length, n = hi - lo;
  int k = 0;
  auto cp = [&](void* d, const void* h, size_t bytes) {
    return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, S->s_up[k++ % kUpStreams]) == cudaSuccess;
  };
  const bool ok = cp(S->d_keys + (size_t)lo * K, S->h_keys + (size_t)lo * K, (size_t)n * K * 4u) &&
                  cp(S->d_vals + (size_t)lo * V, S->h_vals + (size_t)lo * V, (size_t)n * V * 4u) &&
                  cp(S->d_types + lo, S->h_types + lo, n) &&
                  cp(S->d_klens + lo, S->h_klens + lo, (size_t)n * 4u) &&
                  cp(S->d_vlens + lo, S->h_vlens + lo, (size_t)n * 4u) &&
                  cp(S->d_order + lo, S->h_order + lo, (size_t)n * 4u);
  return ok ? MT_OK : MT_ERR_CUDA;
}

// The round's copies on every upload stream are done when this event, recorded
// on the first stream after it waits for the others, has completed.
int server_round_event(mt_server* S, cudaEvent_t ev) {
  for (int k = 1; k < kUpStreams; ++k)
    if (cudaEventRecord(S->up_join[k], S->s_up[k]) != cudaSuccess ||
        cudaStreamWaitEvent(S->s_up[0], S->up_join[k], 0) != cudaSuccess)
      return MT_ERR_CUDA;
  return cudaEventRecord(ev, S->s_up[0]) == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

// Results of a completed request, from the mapped outputs to its buffers:
// find values and value lengths, write results (what mt_mixed_batch writes).
void server_deliver(mt_server* S, const srv_request& r) {
  const uint32_t V = S->cfg.max_value_length, off = r.off;
  for (uint32_t o = 0; o < r.n; ++o) {
    if (r.types[o] == MT_REQ_FIND) {
      const uint32_t vl = S->m_vlens[off + o];
      r.vlens[o] = vl;
      const uint32_t c = std::min(vl, V);
      if (c) std::memcpy(r.vals + (size_t)o * V, S->m_vals + (size_t)(off + o) * V, (size_t)c * 4u);
    } else if (r.results && r.types[o] <= MT_REQ_UPDATE) {
      r.results[o] = S->m_results[off + o];
    }
  }
}

void server_pump(mt_server* S) {
  mt_masstree* t = S->tree;
  if (cudaSetDevice(t->device) != cudaSuccess) {
    S->status = MT_ERR_CUDA;
    S->exited = true;
    return;
  }
  const uint32_t C = S->C, R = S->R;
  const uint32_t tiles_per_warp = 32u / t->tile_size;
  const uint64_t total_tiles = S->nwarps * tiles_per_warp;
  const bool auto_chunk = S->cfg.chunk_ops == 0;
  const uint32_t fixed_chunk = std::max<uint32_t>(1u, std::min<uint32_t>(S->cfg.chunk_ops, 4096u));
  const double budget = S->cfg.memory_budget > 0.f ? S->cfg.memory_budget : 0.9;
  const unsigned long long epoch_ns = (unsigned long long)(S->cfg.epoch_us ? S->cfg.epoch_us : 20000u) * 1000ull;
  const uint32_t per_write = 1u + suf_nodes(S->cfg.max_key_length, S->cfg.max_value_length);
  int rc = MT_OK;
  mt_stats_t st{};
  if (mt_stats(t, &st) != MT_OK) rc = MT_ERR_CUDA;
  const double slab_budget = budget * (double)st.total_slabs;
  double slabs_in_use = (double)st.used_slabs + (double)st.limbo_slabs;
  uint64_t admitted_demand = 0, completed_demand = 0;

  std::deque<uint32_t> fifo;      // slots in admission order (frees staging)
  std::deque<srv_round> rounds;   // upload rounds in flight, in order
  std::vector<uint32_t> published, finished_now;
  uint64_t head = 0, tail = 0;    // staging ring (ops)
  uint64_t items_published = 0, admitted_ops = 0, completed_ops = 0;
  std::vector<cudaEvent_t> evs;
  std::vector<uint64_t> enq_completed;
  size_t ev_done = 0;
  auto take_event = [&]() -> cudaEvent_t {
    if (!S->ev_pool.empty()) {
      cudaEvent_t e = S->ev_pool.back();
      S->ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
  };
  auto enqueue_epoch = [&]() -> int {
    int r2 = host_launch_reclaim(t, S->s_work);
    if (r2) return r2;
    pool_usage_kernel<<<1, 32, 0, S->s_work>>>(t->tv.pool, S->d_usage);
    r2 = launch_server_tile(t, S->blocks, S->sv, epoch_ns, S->s_work);
    if (r2) return r2;
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MT_ERR_CUDA;
    if (cudaEventRecord(e, S->s_work) != cudaSuccess) return MT_ERR_CUDA;
    evs.push_back(e);
    enq_completed.push_back(completed_demand);
    return MT_OK;
  };
  if (!rc) rc = enqueue_epoch();
  if (!rc) rc = enqueue_epoch();
  uint64_t stuck_since = 0;
  while (!rc) {
    bool progress = false;
    // ---- admit queued requests in order, staged and uploaded together ------
    srv_round round;
    uint64_t round_ops = 0;
    uint32_t run_lo = 0, run_hi = 0;  // current contiguous staging run
    bool have_run = false;
    const uint64_t round_ns = now_ns(S->t0);
    while (!rc) {
      srv_request r;
      {
        std::lock_guard<std::mutex> g(S->mu);
        if (S->queued.empty() || round_ops >= kRoundMaxOps) break;
        const srv_request& f = S->queued.front();
        const uint64_t oldest = fifo.empty() ? f.ticket : S->slots[fifo.front()].ticket;
        if (f.ticket - oldest >= R) break;  // no free request slot
        uint64_t h = head;
        if (h % C + f.n > C) h += C - h % C;  // the request's ops stay contiguous
        if (h + f.n - tail > C) break;        // no staging space
        uint32_t d = 0;
        for (uint32_t o = 0; o < f.n; ++o)
          d += (f.types[o] == MT_REQ_INSERT || f.types[o] == MT_REQ_UPDATE) ? per_write : 0u;
        if (slabs_in_use + d > slab_budget) {
          // Admission waits for memory (slabs come back between launches).
          if (fifo.empty()) {
            const uint64_t now = now_ns(S->t0);
            if (!stuck_since) stuck_since = now;
            else if (now - stuck_since > 60ull * 1000000000ull) rc = MT_ERR_OOM;  // never fits
          }
          break;
        }
        stuck_since = 0;
        r = f;
        S->queued.pop_front();
        r.off = (uint32_t)(h % C);
        head = h + r.n;
        r.alloc_end = head;
        r.demand = d;
      }
      const uint32_t slot = (uint32_t)(r.ticket % R);
      r.stage = SRV_UPLOADING;
      r.admit_ns = round_ns;
      S->slots[slot] = r;
      const uint32_t rec = (uint32_t)(r.ticket % S->L);
      S->rec_done[rec].store(0u, std::memory_order_relaxed);
      S->rec_ticket[rec].store(r.ticket, std::memory_order_release);
      slabs_in_use += r.demand;
      admitted_demand += r.demand;
      admitted_ops += r.n;
      round_ops += r.n;
      fifo.push_back(slot);
      round.slots.push_back(slot);
      progress = true;
    }
    if (!rc && !round.slots.empty()) {
      // Copy the round's requests into the staging (in parallel when large),
      // then upload each contiguous run of it with one copy per field.
      auto stage = [&](size_t k) { server_stage(S, S->slots[round.slots[k]]); };
      if (round_ops >= kPoolMinOps) S->pool.run(round.slots.size(), stage);
      else for (size_t k = 0; k < round.slots.size(); ++k) stage(k);
      for (uint32_t slot : round.slots) {
        const srv_request& q = S->slots[slot];
        if (have_run && q.off == run_hi) {
          run_hi += q.n;
        } else {
          if (have_run && !rc) rc = server_upload_range(S, run_lo, run_hi);
          run_lo = q.off;
          run_hi = q.off + q.n;
          have_run = true;
        }
      }
      if (!rc) rc = server_upload_range(S, run_lo, run_hi);
      round.ev = take_event();
      if (!round.ev) rc = MT_ERR_CUDA;
      if (!rc) rc = server_round_event(S, round.ev);
      if (!rc) rounds.push_back(std::move(round));
    }
    // ---- publish uploaded rounds as work items --------------------------------
    while (!rc && !rounds.empty() && cudaEventQuery(rounds.front().ev) == cudaSuccess) {
      srv_round& rd = rounds.front();
      const uint64_t pub_ns = now_ns(S->t0);
      for (uint32_t slot : rd.slots) {
        srv_request& q = S->slots[slot];
        uint32_t chunk = fixed_chunk;
        if (auto_chunk) {
          const uint64_t backlog = admitted_ops - std::min(admitted_ops, completed_ops);
          const uint64_t per_tile = backlog / total_tiles;
          chunk = backlog < S->nwarps / 8 ? 1u
                                           : tiles_per_warp * (per_tile < 1 ? 1u : per_tile < 2 ? 2u : per_tile < 4 ? 4u : 8u);
        }
        const uint32_t n_items = std::max<uint32_t>(1u, (q.n + chunk - 1) / chunk);
        S->done[slot] = 0u;
        uint32_t f = q.off, left = q.n;
        for (uint32_t k = 0; k < n_items; ++k) {
          const uint32_t c = std::min(left, chunk);
          S->ring[items_published % C] = serve_item{slot, f, c, n_items};
          ++items_published;
          f += c;
          left -= c;
        }
        q.stage = SRV_PUBLISHED;
        q.publish_ns = pub_ns;
        published.push_back(slot);
      }
      __atomic_store_n(S->pub, (unsigned long long)items_published, __ATOMIC_RELEASE);
      S->ev_pool.push_back(rd.ev);
      rounds.pop_front();
      progress = true;
    }
    // ---- completed on the device: deliver the results -------------------------
    finished_now.clear();
    uint64_t finished_ops = 0;
    const uint64_t seen_ns = published.empty() ? 0 : now_ns(S->t0);
    for (size_t k = 0; !rc && k < published.size();) {
      const uint32_t slot = published[k];
      if (__atomic_load_n(&S->done[slot], __ATOMIC_ACQUIRE)) {
        S->slots[slot].done_ns = seen_ns;
        finished_now.push_back(slot);
        finished_ops += S->slots[slot].n;
        published[k] = published.back();
        published.pop_back();
      } else {
        ++k;
      }
    }
    if (!finished_now.empty()) {
      auto deliver = [&](size_t k) { server_deliver(S, S->slots[finished_now[k]]); };
      if (finished_ops >= kPoolMinOps) S->pool.run(finished_now.size(), deliver);
      else for (size_t k = 0; k < finished_now.size(); ++k) deliver(k);
      const uint64_t now = now_ns(S->t0);
      uint64_t sq = 0, su = 0, sd = 0, sl = 0, mx = 0;
      for (uint32_t slot : finished_now) {
        srv_request& q = S->slots[slot];
        q.stage = SRV_DONE;
        completed_demand += q.demand;
        completed_ops += q.n;
        const uint32_t rec = (uint32_t)(q.ticket % S->L);
        S->rec_latency[rec].store(now - q.submit_ns, std::memory_order_relaxed);
        S->rec_done[rec].store(1u, std::memory_order_release);
        sq += q.admit_ns - std::min(q.admit_ns, q.submit_ns);
        su += q.publish_ns - q.admit_ns;
        sd += q.done_ns - q.publish_ns;
        sl += now - q.done_ns;
        mx = std::max(mx, now - q.submit_ns);
      }
      S->st_queued.fetch_add(sq, std::memory_order_relaxed);
      S->st_upload.fetch_add(su, std::memory_order_relaxed);
      S->st_device.fetch_add(sd, std::memory_order_relaxed);
      S->st_deliver.fetch_add(sl, std::memory_order_relaxed);
      S->st_ops.fetch_add(finished_ops, std::memory_order_relaxed);
      if (mx > S->st_max.load(std::memory_order_relaxed)) S->st_max.store(mx, std::memory_order_relaxed);
      S->st_requests.fetch_add(finished_now.size(), std::memory_order_release);
      progress = true;
    }
    while (!fifo.empty() && S->slots[fifo.front()].stage == SRV_DONE) {
      tail = std::max(tail, S->slots[fifo.front()].alloc_end);
      fifo.pop_front();
    }
    // ---- keep the device loop running -------------------------------------------
    while (!rc && ev_done < evs.size() && cudaEventQuery(evs[ev_done]) == cudaSuccess) {
      ++ev_done;
      rc = enqueue_epoch();
      // Retired slabs came back with the reclaim pass before that launch:
      // restart the estimate from the pool count taken then, plus the demand
      // of every request not complete when that epoch was enqueued.
      slabs_in_use = (double)__atomic_load_n(S->usage, __ATOMIC_ACQUIRE) +
                     (double)(admitted_demand - std::min(admitted_demand, enq_completed[ev_done - 1]));
      if (ev_done > 64) {  // events of finished epochs
        for (size_t k = 0; k + 2 < ev_done; ++k) cudaEventDestroy(evs[k]);
        evs.erase(evs.begin(), evs.begin() + (ev_done - 2));
        enq_completed.erase(enq_completed.begin(), enq_completed.begin() + (ev_done - 2));
        ev_done = 2;
      }
    }
    if (S->quit.load(std::memory_order_acquire)) break;
    if (S->draining.load(std::memory_order_acquire) && fifo.empty()) {
      std::lock_guard<std::mutex> g(S->mu);
      if (S->queued.empty()) break;
    }
    if (!progress) std::this_thread::yield();
  }
  // The device loop leaves at the stop flag (or its launch's time budget).
  __atomic_store_n(S->stop, 1u, __ATOMIC_RELEASE);
  cudaStreamSynchronize(S->s_work);
  for (cudaStream_t st : S->s_up) cudaStreamSynchronize(st);
  for (auto& rd : rounds) S->ev_pool.push_back(rd.ev);
  for (auto e : evs) cudaEventDestroy(e);
  if (rc) S->status = rc;
  S->exited.store(true, std::memory_order_release);
}

}  // namespace

extern "C" int mt_server_start(mt_masstree* t, const mt_server_config* cfg, mt_server** out) {
  if (!t || !cfg || !out || cfg->max_key_length == 0 || cfg->max_value_length == 0) return MT_ERR_INVALID_ARG;
  *out = nullptr;
  if (cudaSetDevice(t->device) != cudaSuccess) return MT_ERR_CUDA;
  auto* S = new (std::nothrow) mt_server();
  if (!S) return MT_ERR_OOM;
  S->tree = t;
  S->cfg = *cfg;
  S->C = cfg->max_ops_in_flight ? cfg->max_ops_in_flight : (1u << 20);
  S->R = cfg->max_requests_in_flight ? cfg->max_requests_in_flight : 65536u;
  S->L = std::max<uint32_t>(S->R, 65536u);
  const uint32_t C = S->C, R = S->R, K = cfg->max_key_length, V = cfg->max_value_length;
  auto up = [](size_t b) { return (b + 255u) & ~size_t(255); };
  const size_t bytes = up(C) + up((size_t)C * K * 4u) + 3 * up((size_t)C * 4u) + up((size_t)C * V * 4u);
  bool ok = cudaMalloc(&S->dmem, bytes) == cudaSuccess && cudaMallocHost(&S->hmem, bytes) == cudaSuccess;
  if (ok) {
    char* p = static_cast<char*>(S->dmem);
    char* h = static_cast<char*>(S->hmem);
    auto carve = [&](size_t b, auto** dptr, auto** hptr) {
      *dptr = reinterpret_cast<std::remove_pointer_t<decltype(dptr)>>(p);
      *hptr = reinterpret_cast<std::remove_pointer_t<decltype(hptr)>>(h);
      p += up(b);
      h += up(b);
    };
    carve(C, &S->d_types, &S->h_types);
    carve((size_t)C * K * 4u, &S->d_keys, &S->h_keys);
    carve((size_t)C * 4u, &S->d_klens, &S->h_klens);
    carve((size_t)C * 4u, &S->d_vlens, &S->h_vlens);
    carve((size_t)C * 4u, &S->d_order, &S->h_order);
    carve((size_t)C * V * 4u, &S->d_vals, &S->h_vals);
  }
  if (ok) {
    S->m_vals = mapped_alloc<uint32_t>((size_t)C * V, &S->m_vals_d);
    S->m_vlens = mapped_alloc<uint32_t>(C, &S->m_vlens_d);
    S->m_results = mapped_alloc<bool>(C, &S->m_results_d);
    S->ring = mapped_alloc<serve_item>(C, &S->d_ring);
    S->pub = mapped_alloc<unsigned long long>(1, &S->d_pub);
    S->stop = mapped_alloc<uint32_t>(1, &S->d_stop);
    S->done = mapped_alloc<uint32_t>(R, &S->d_done);
    S->usage = mapped_alloc<unsigned long long>(1, &S->d_usage);
    ok = S->m_vals && S->m_vlens && S->m_results && S->ring && S->pub && S->stop && S->done && S->usage;
  }
  S->blocks = server_blocks_tile(t);
  S->nwarps = (size_t)S->blocks * (kBlock / 32);
  ok = ok && cudaMalloc(&S->d_finished, (size_t)R * 4u) == cudaSuccess &&
       cudaMemset(S->d_finished, 0, (size_t)R * 4u) == cudaSuccess &&
       cudaMalloc(&S->d_ctl, sizeof(server_ctl)) == cudaSuccess &&
       cudaMemset(S->d_ctl, 0, sizeof(server_ctl)) == cudaSuccess &&
       cudaMalloc(&S->d_held, S->nwarps * sizeof(unsigned long long)) == cudaSuccess &&
       cudaMemset(S->d_held, 0xFF, S->nwarps * sizeof(unsigned long long)) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&S->s_work, cudaStreamNonBlocking) == cudaSuccess &&
       [&] {
         for (int k = 0; k < kUpStreams; ++k)
           if (cudaStreamCreateWithFlags(&S->s_up[k], cudaStreamNonBlocking) != cudaSuccess ||
               cudaEventCreateWithFlags(&S->up_join[k], cudaEventDisableTiming) != cudaSuccess)
             return false;
         return true;
       }();
  if (ok) {
    S->slots.resize(R);
    S->rec_ticket.reset(new (std::nothrow) std::atomic<uint64_t>[S->L]);
    S->rec_done.reset(new (std::nothrow) std::atomic<uint32_t>[S->L]);
    S->rec_latency.reset(new (std::nothrow) std::atomic<uint64_t>[S->L]);
    ok = S->rec_ticket && S->rec_done && S->rec_latency;
    for (uint32_t k = 0; ok && k < S->L; ++k) {
      S->rec_ticket[k].store(0);
      S->rec_done[k].store(0);
      S->rec_latency[k].store(0);
    }
  }
  if (!ok) {
    server_free(S);
    return MT_ERR_OOM;
  }
  server_view& sv = S->sv;
  sv.ring = S->d_ring;
  sv.published = S->d_pub;
  sv.stop = S->d_stop;
  sv.ctl = S->d_ctl;
  sv.held = S->d_held;
  sv.finished = S->d_finished;
  sv.done = S->d_done;
  sv.ring_cap = C;
  sv.order = S->d_order;
  batch_args ops{};
  ops.types = S->d_types;
  ops.keys = S->d_keys;
  ops.key_lengths = S->d_klens;
  ops.values = S->d_vals;            // insert and update values
  ops.values_out = S->m_vals_d;      // find values, to mapped host memory
  ops.value_lengths_in = S->d_vlens;
  ops.value_lengths_out = S->m_vlens_d;
  ops.results = S->m_results_d;
  ops.max_key_length = K;
  ops.max_value_length = V;
  sv.ops = ops;
  // Every earlier call on the tree finishes first; one launch without a time
  // budget loads the kernel and leaves every warp holding its first ticket.
  *S->usage = 0;
  ok = cudaDeviceSynchronize() == cudaSuccess && host_launch_reclaim(t, S->s_work) == MT_OK &&
       launch_server_tile(t, S->blocks, sv, 0ull, S->s_work) == MT_OK &&
       cudaStreamSynchronize(S->s_work) == cudaSuccess;
  if (!ok) {
    server_free(S);
    return MT_ERR_CUDA;
  }
  S->t0 = clk::now();
  S->pool.start((int)std::min(6u, std::max(1u, std::thread::hardware_concurrency() / 4u)));
  S->pump = std::thread(server_pump, S);
  *out = S;
  return MT_OK;
}

extern "C" int mt_server_submit(mt_server* S, const uint8_t* types, const uint32_t* keys, const uint32_t* klens,
                                uint32_t* vals, uint32_t* vlens, bool* results, uint32_t n, uint64_t* ticket) {
  if (!S || !ticket || n == 0 || n > S->C || !types || !keys || !vals || !vlens) return MT_ERR_INVALID_ARG;
  if (S->draining.load(std::memory_order_acquire)) return MT_ERR_INVALID_ARG;
  const int st = S->status.load(std::memory_order_acquire);
  if (st) return st;
  srv_request r;
  r.types = types;
  r.keys = keys;
  r.klens = klens;
  r.vals = vals;
  r.vlens = vlens;
  r.results = results;
  r.n = n;
  std::lock_guard<std::mutex> g(S->mu);
  r.submit_ns = now_ns(S->t0);
  r.ticket = S->next_ticket.load(std::memory_order_relaxed);
  S->queued.push_back(r);
  S->next_ticket.store(r.ticket + 1, std::memory_order_release);
  *ticket = r.ticket;
  return MT_OK;
}

extern "C" int mt_server_poll(mt_server* S, uint64_t ticket, int* done, uint64_t* latency_ns) {
  if (!S || !done || ticket >= S->next_ticket.load(std::memory_order_acquire)) return MT_ERR_INVALID_ARG;
  const uint32_t rec = (uint32_t)(ticket % S->L);
  const uint64_t rt = S->rec_ticket[rec].load(std::memory_order_acquire);
  *done = 0;
  if (latency_ns) *latency_ns = 0;
  if (rt > ticket) {
    *done = 1;  // the record moved on to a later request: this one completed (its latency is gone)
  } else if (rt == ticket && S->rec_done[rec].load(std::memory_order_acquire)) {
    *done = 1;
    if (latency_ns) *latency_ns = S->rec_latency[rec].load(std::memory_order_relaxed);
  }
  if (!*done) {
    const int st = S->status.load(std::memory_order_acquire);
    if (st) return st;
  }
  return MT_OK;
}

extern "C" int mt_server_stats(mt_server* S, mt_server_stats_t* out) {
  if (!S || !out) return MT_ERR_INVALID_ARG;
  *out = mt_server_stats_t{};
  out->requests = S->st_requests.load(std::memory_order_acquire);
  out->ops = S->st_ops.load(std::memory_order_relaxed);
  out->queued_ns = S->st_queued.load(std::memory_order_relaxed);
  out->upload_ns = S->st_upload.load(std::memory_order_relaxed);
  out->device_ns = S->st_device.load(std::memory_order_relaxed);
  out->deliver_ns = S->st_deliver.load(std::memory_order_relaxed);
  out->max_latency_ns = S->st_max.load(std::memory_order_relaxed);
  return MT_OK;
}

extern "C" int mt_server_stop(mt_server* S) {
  if (!S) return MT_ERR_INVALID_ARG;
  // Serve what is queued; bound the wait, then end the loop regardless.
  S->draining.store(true, std::memory_order_release);
  const auto deadline = clk::now() + std::chrono::seconds(60);
  while (!S->exited.load(std::memory_order_acquire) && clk::now() < deadline)
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  const bool drained = S->exited.load(std::memory_order_acquire);
  S->quit.store(true, std::memory_order_release);
  if (S->pump.joinable()) S->pump.join();
  int rc = S->status.load();
  if (!rc && !drained) rc = MT_ERR_LOCK_TIMEOUT;
  mt_masstree* t = S->tree;
  server_free(S);
  const int dev_rc = mt_sync(t, nullptr);
  return rc ? rc : dev_rc;
}

namespace {

// MT_SERVE_ONLINE: replay of an open-loop plan through mt_server_*.  Requests
// are submitted in arrival order, each when its arrival time has come, from
// host buffers; a poller thread records when each one is done.  Latency is
// done - arrival (the submit call, the upload, the device work and the
// download of the results).
int serve_online(mt_masstree* t, const mt_serve_plan* plan, uint64_t* latency_ns, mt_serve_stats* stats) {
  const uint32_t nreq = plan->num_requests;
  uint32_t max_ops = 1;
  for (uint32_t r = 0; r < nreq; ++r) {
    if (r > 0 && plan->arrival_ns[r] < plan->arrival_ns[r - 1]) return MT_ERR_INVALID_ARG;
    if (plan->request_num_ops[r] == 0) return MT_ERR_INVALID_ARG;
    max_ops = std::max(max_ops, plan->request_num_ops[r]);
  }
  mt_server_config cfg{};
  cfg.max_key_length = plan->max_key_length;
  cfg.max_value_length = plan->max_value_length;
  cfg.max_ops_in_flight = std::max<uint32_t>(1u << 20, max_ops);
  cfg.chunk_ops = plan->chunk_ops;
  cfg.epoch_us = plan->epoch_us;
  cfg.memory_budget = plan->memory_budget;
  mt_server* S = nullptr;
  int rc = mt_server_start(t, &cfg, &S);
  if (rc) return rc;
  std::vector<uint64_t> tickets(nreq, ~0ull), submitted(nreq, 0), completion(nreq, 0);
  std::atomic<uint32_t> n_submitted{0};
  std::atomic<bool> submit_end{false};
  std::atomic<bool> poll_fail{false};
  const clk::time_point t0 = clk::now();
  std::thread poller([&] {
    uint32_t next = 0;
    std::vector<uint32_t> pending;
    while (true) {
      const bool ended = submit_end.load(std::memory_order_acquire);
      const uint32_t ns = n_submitted.load(std::memory_order_acquire);
      if (ended && next == ns && pending.empty()) break;
      while (next < ns) pending.push_back(next++);
      bool progress = false;
      for (size_t k = 0; k < pending.size();) {
        int d = 0;
        if (mt_server_poll(S, tickets[pending[k]], &d, nullptr) != MT_OK) {
          poll_fail = true;
          return;
        }
        if (d) {
          completion[pending[k]] = now_ns(t0);
          pending[k] = pending.back();
          pending.pop_back();
          progress = true;
        } else {
          ++k;
        }
      }
      if (now_ns(t0) > plan->arrival_ns[nreq - 1] + 60ull * 1000000000ull) {
        poll_fail = true;
        return;
      }
      if (!progress) std::this_thread::yield();
    }
  });
  for (uint32_t r = 0; r < nreq && !rc && !poll_fail; ++r) {
    while (now_ns(t0) < plan->arrival_ns[r]) {
    }
    const uint32_t f = plan->request_first_op[r], n = plan->request_num_ops[r];
    rc = mt_server_submit(S, plan->types + f, plan->keys + (size_t)f * plan->max_key_length,
                          plan->key_lengths ? plan->key_lengths + f : nullptr,
                          plan->values + (size_t)f * plan->max_value_length, plan->value_lengths + f,
                          plan->results ? plan->results + f : nullptr, n, &tickets[r]);
    submitted[r] = now_ns(t0);
    if (!rc) n_submitted.store(r + 1, std::memory_order_release);
  }
  submit_end.store(true, std::memory_order_release);
  poller.join();
  mt_server_stats_t sst{};
  mt_server_stats(S, &sst);
  const int stop_rc = mt_server_stop(S);
  uint64_t ops_done = 0, end = 0, done_req = 0;
  for (uint32_t r = 0; r < nreq; ++r) {
    latency_ns[r] = completion[r] ? completion[r] - std::min(completion[r], plan->arrival_ns[r]) : 0ull;
    if (completion[r]) {
      ops_done += plan->request_num_ops[r];
      ++done_req;
    }
    end = std::max<uint64_t>(end, completion[r]);
  }
  if (stats) {
    stats->wall_ns = end;
    stats->requests_done = done_req;
    stats->ops_done = ops_done;
    stats->admission_waits = 0;
    stats->stage_ns[0] = sst.queued_ns;
    stats->stage_ns[1] = sst.upload_ns;
    stats->stage_ns[2] = sst.device_ns;
    stats->stage_ns[3] = sst.deliver_ns;
  }
  if (!rc && poll_fail) rc = MT_ERR_LOCK_TIMEOUT;
  return rc ? rc : stop_rc;
}

}  // namespace
