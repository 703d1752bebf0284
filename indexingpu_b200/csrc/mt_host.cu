// Mixed batches from host buffers with copy/compute overlap (mt_mixed_batch_host).
//
// The reference's host API takes device buffers (include/gpu_masstree.hpp:173-191);
// a caller holding requests in host memory copies them in, calls, and copies the
// results out, one step after the other.  This entry point does the copies
// itself, overlapped with the work: the batch is cut into chunks that go
// through a ring of device staging slots, inputs on an upload stream, results
// on a download stream, each chunk served as one mt_mixed_batch on the
// caller's stream.  While chunk j runs, chunk j+1 is uploaded and chunk j-1
// downloaded, within one call and across consecutive calls.  A mixed batch has
// no order among its requests, so serving it as consecutive chunks is one of
// its allowed orders.
#include <algorithm>

#include "mt_internal.cuh"

using namespace mtb;

namespace {

constexpr int kSlots = 3;
constexpr uint32_t kDefaultChunk = 1u << 18;

struct host_slot {
  uint8_t* types = nullptr;
  uint32_t* keys = nullptr;
  uint32_t* klens = nullptr;
  uint32_t* vals = nullptr;
  uint32_t* vlens = nullptr;
  bool* results = nullptr;
  cudaEvent_t uploaded = nullptr;    // inputs of the slot's current chunk are on the device
  cudaEvent_t served = nullptr;      // its chunk has been served
  cudaEvent_t downloaded = nullptr;  // its results are back in host memory (slot free)
  bool used = false;
};

}  // namespace

struct mt_host_pipe {
  void* mem = nullptr;
  uint32_t chunk = 0, max_k = 0, max_v = 0;
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t inputs_ready = nullptr;  // MT_FLAG_INPUTS_ON_STREAM: the caller's stream reached the call
  host_slot slot[kSlots];
  uint64_t next = 0;  // chunks issued so far (slot = next % kSlots)
};

namespace mtb {

void host_pipe_free(mt_masstree* t) {
  mt_host_pipe* hp = t->host_pipe;
  if (!hp) return;
  if (hp->mem) cudaFree(hp->mem);
  for (auto& s : hp->slot) {
    if (s.uploaded) cudaEventDestroy(s.uploaded);
    if (s.served) cudaEventDestroy(s.served);
    if (s.downloaded) cudaEventDestroy(s.downloaded);
  }
  if (hp->inputs_ready) cudaEventDestroy(hp->inputs_ready);
  if (hp->up) cudaStreamDestroy(hp->up);
  if (hp->down) cudaStreamDestroy(hp->down);
  delete hp;
  t->host_pipe = nullptr;
}

}  // namespace mtb

namespace {

// Staging for chunks of `chunk` requests of the given row strides (allocates:
// on first use and when a call needs longer rows or larger chunks).
int ensure_pipe(mt_masstree* t, uint32_t chunk, uint32_t max_k, uint32_t max_v) {
  mt_host_pipe* hp = t->host_pipe;
  if (hp && hp->chunk >= chunk && hp->max_k >= max_k && hp->max_v >= max_v) return MT_OK;
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  if (hp) {
    chunk = std::max(chunk, hp->chunk);
    max_k = std::max(max_k, hp->max_k);
    max_v = std::max(max_v, hp->max_v);
    host_pipe_free(t);
  }
  hp = new (std::nothrow) mt_host_pipe();
  if (!hp) return MT_ERR_OOM;
  t->host_pipe = hp;
  auto up16 = [](size_t b) { return (b + 255u) & ~size_t(255); };
  const size_t c = chunk;
  const size_t per_slot = up16(c) + up16(c * max_k * 4u) + up16(c * 4u) + up16(c * max_v * 4u) + up16(c * 4u) +
                          up16(c);
  if (cudaMalloc(&hp->mem, per_slot * kSlots) != cudaSuccess) {
    host_pipe_free(t);
    return MT_ERR_OOM;
  }
  hp->chunk = chunk;
  hp->max_k = max_k;
  hp->max_v = max_v;
  char* p = static_cast<char*>(hp->mem);
  bool ok = cudaStreamCreateWithFlags(&hp->up, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&hp->down, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&hp->inputs_ready, cudaEventDisableTiming) == cudaSuccess;
  for (auto& s : hp->slot) {
    s.types = reinterpret_cast<uint8_t*>(p);
    p += up16(c);
    s.keys = reinterpret_cast<uint32_t*>(p);
    p += up16(c * max_k * 4u);
    s.klens = reinterpret_cast<uint32_t*>(p);
    p += up16(c * 4u);
    s.vals = reinterpret_cast<uint32_t*>(p);
    p += up16(c * max_v * 4u);
    s.vlens = reinterpret_cast<uint32_t*>(p);
    p += up16(c * 4u);
    s.results = reinterpret_cast<bool*>(p);
    p += up16(c);
    ok = ok && cudaEventCreateWithFlags(&s.uploaded, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&s.served, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&s.downloaded, cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    host_pipe_free(t);
    return MT_ERR_CUDA;
  }
  return MT_OK;
}

int copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  if (bytes == 0) return MT_OK;
  return cudaMemcpyAsync(dst, src, bytes, kind, s) == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

}  // namespace

extern "C" int mt_mixed_batch_host(mt_masstree* t, const uint8_t* types, const uint32_t* keys, uint32_t maxK,
                                   const uint32_t* klens, uint32_t* values, uint32_t maxV, uint32_t* vlens,
                                   bool* results, uint32_t n, uint32_t chunk, uint32_t flags, void* stream) {
  if (!t || (n && (!types || !keys || !values || !vlens || maxK == 0 || maxV == 0))) return MT_ERR_INVALID_ARG;
  if (n == 0) return MT_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (chunk == 0) chunk = kDefaultChunk;
  chunk = std::min(chunk, n);
  int rc = ensure_pipe(t, chunk, maxK, maxV);
  if (rc) return rc;
  mt_host_pipe* hp = t->host_pipe;
  if (flags & MT_FLAG_INPUTS_ON_STREAM) {
    // The inputs are produced by work already queued on the caller's stream.
    if (cudaEventRecord(hp->inputs_ready, s) != cudaSuccess ||
        cudaStreamWaitEvent(hp->up, hp->inputs_ready, 0) != cudaSuccess)
      return MT_ERR_CUDA;
  }
  flags &= ~MT_FLAG_INPUTS_ON_STREAM;
  // Rows keep the caller's strides inside a slot (its rows are at least as long).
  for (uint32_t first = 0; first < n; first += chunk) {
    const uint32_t m = std::min(chunk, n - first);
    host_slot& sl = hp->slot[hp->next % kSlots];
    ++hp->next;
    // Upload once the slot's previous chunk is back in host memory (its
    // download follows its service, the only reader of the slot).
    if (sl.used && cudaStreamWaitEvent(hp->up, sl.downloaded, 0) != cudaSuccess) return MT_ERR_CUDA;
    rc = copy(sl.types, types + first, m, cudaMemcpyHostToDevice, hp->up);
    if (!rc) rc = copy(sl.keys, keys + (size_t)first * maxK, (size_t)m * maxK * 4u, cudaMemcpyHostToDevice, hp->up);
    if (!rc && klens) rc = copy(sl.klens, klens + first, (size_t)m * 4u, cudaMemcpyHostToDevice, hp->up);
    if (!rc) rc = copy(sl.vals, values + (size_t)first * maxV, (size_t)m * maxV * 4u, cudaMemcpyHostToDevice, hp->up);
    if (!rc) rc = copy(sl.vlens, vlens + first, (size_t)m * 4u, cudaMemcpyHostToDevice, hp->up);
    if (rc) return rc;
    if (cudaEventRecord(sl.uploaded, hp->up) != cudaSuccess) return MT_ERR_CUDA;
    // Serve the chunk on the caller's stream, after the batches before it.
    if (cudaStreamWaitEvent(s, sl.uploaded, 0) != cudaSuccess) return MT_ERR_CUDA;
    rc = mt_mixed_batch(t, sl.types, sl.keys, maxK, klens ? sl.klens : nullptr, sl.vals, maxV, sl.vlens,
                        results ? sl.results : nullptr, m, flags, s);
    if (rc) return rc;
    if (cudaEventRecord(sl.served, s) != cudaSuccess) return MT_ERR_CUDA;
    // Download find values and lengths and the per-request results.
    if (cudaStreamWaitEvent(hp->down, sl.served, 0) != cudaSuccess) return MT_ERR_CUDA;
    rc = copy(values + (size_t)first * maxV, sl.vals, (size_t)m * maxV * 4u, cudaMemcpyDeviceToHost, hp->down);
    if (!rc) rc = copy(vlens + first, sl.vlens, (size_t)m * 4u, cudaMemcpyDeviceToHost, hp->down);
    if (!rc && results) rc = copy(results + first, sl.results, m, cudaMemcpyDeviceToHost, hp->down);
    if (rc) return rc;
    if (cudaEventRecord(sl.downloaded, hp->down) != cudaSuccess) return MT_ERR_CUDA;
    sl.used = true;
    // The call completes on s: s waits for the last chunk's results.
    if (first + m >= n && cudaStreamWaitEvent(s, sl.downloaded, 0) != cudaSuccess) return MT_ERR_CUDA;
  }
  return MT_OK;
}
