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
#include <cstring>
#include <thread>
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
    serve_requests<T, OP_MIXED, true>(t, tv, cache, a, tile_in_warp, tiles_per_warp);
    __syncwarp();
    if (lane == 0) {
      // acq_rel: the last item of a request has seen every write of the
      // others, all in device memory, before it raises the request's flag
      // (the host reads results only through later copies or calls).
      const uint32_t f = atom_add_acq_rel_gpu_u32(sv.finished + it.req, 1u) + 1u;
      if (f == it.items) st_relaxed_sys_u32(sv.done + it.req, 1u);
      else if (f > it.items) record_error(tv.pool, ERR_CORRUPT);  // an item served twice
    }
    // Warp-uniform: lane 0 reads the clock and decides for the whole warp
    // (every lane's own reading could split the warp).
    if (__shfl_sync(0xFFFFFFFFu, (lane == 0 && global_ns() > deadline) ? 1u : 0u, 0)) break;
  }
  if (lane == 0) sv.held[wid] = keep;
  cache.release(t, tv.pool);
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

extern "C" int mt_serve(mt_masstree* t, const mt_serve_plan* plan, uint64_t* latency_ns, mt_serve_stats* stats) {
  if (!t || !plan || !latency_ns || plan->num_requests == 0 || !plan->request_first_op || !plan->request_num_ops ||
      !plan->arrival_ns || !plan->types || !plan->keys || !plan->values || !plan->value_lengths ||
      plan->max_key_length == 0 || plan->max_value_length == 0 ||
      (plan->mode != MT_SERVE_SERVED && plan->mode != MT_SERVE_PLAIN))
    return MT_ERR_INVALID_ARG;
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
  }
  if (!rc) rc = mt_sync(t, nullptr);
  return rc;
}
