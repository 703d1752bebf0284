// Tile and memory primitives for the B200 masstree.
//
// A "tile" is a group of T consecutive lanes of one warp (T = 4, 8, 16 or 32)
// that serves one request at a time.  A 128-byte node is held by the tile with
// W = 32 / T words per lane, loaded and stored with ONE vector instruction per
// lane (v8 = 32 B at T=4, v4 at T=8, v2 at T=16, scalar at T=32), so a node is
// always one fully coalesced 128-byte line access.
//
// The reference's tiles are 16 or 32 lanes with 8 or 4 bytes per lane
// (include/utils.hpp:163-260, include/masstree_node_subwarp.hpp:87-121); the
// smaller tiles here exist to put more independent descents in flight per SM.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MT_DEV __device__ __forceinline__
#define MT_HD __host__ __device__ __forceinline__

namespace mtb {

template <int T>
struct tile {
  static_assert(T == 4 || T == 8 || T == 16 || T == 32, "tile size must be 4, 8, 16 or 32");
  static constexpr int size = T;
  static constexpr int W = 32 / T;  // node words held per lane
  uint32_t rank;  // lane index inside the tile
  uint32_t base;  // first warp lane of the tile
  uint32_t mask;  // warp lane mask of the tile

  MT_DEV tile() : tile(threadIdx.x & 31u) {}  // 1-D blocks: lane = threadIdx.x % 32
  // From the warp lane (any block shape: pass %laneid).
  MT_DEV explicit tile(uint32_t wl) {
    rank = wl % T;
    base = wl - rank;
    mask = (T == 32) ? 0xFFFFFFFFu : (((1u << T) - 1u) << base);
  }
  MT_DEV uint32_t shfl(uint32_t v, int src) const { return __shfl_sync(mask, v, src, T); }
  MT_DEV uint64_t shfl64(uint64_t v, int src) const { return __shfl_sync(mask, v, src, T); }
  MT_DEV uint32_t shfl_up(uint32_t v, int d) const { return __shfl_up_sync(mask, v, d, T); }
  MT_DEV uint32_t shfl_down(uint32_t v, int d) const { return __shfl_down_sync(mask, v, d, T); }
  MT_DEV uint32_t ballot(bool p) const { return __ballot_sync(mask, p) >> base; }
  MT_DEV uint32_t or_all(uint32_t v) const { return __reduce_or_sync(mask, v); }
  MT_DEV uint32_t add_all(uint32_t v) const { return __reduce_add_sync(mask, v); }
  MT_DEV uint32_t min_all(uint32_t v) const { return __reduce_min_sync(mask, v); }
  MT_DEV bool any(bool p) const { return ballot(p) != 0u; }
  MT_DEV void sync() const { __syncwarp(mask); }
  MT_DEV bool leader() const { return rank == 0; }
};

MT_DEV uint32_t lane_id() {
  uint32_t l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// Memory orders for node traffic.
//   NC      : read-only path (no writer in the same launch); texture/L1 path.
//   RELAXED : gpu-scope relaxed, served from L2 (coherent), no fence.
//   ACQUIRE : gpu-scope acquire.
enum class ld_order { NC, RELAXED, ACQUIRE };
enum class st_order { WEAK, RELEASE };

template <int W, ld_order O>
MT_DEV void load_words(const uint32_t* p, uint32_t (&w)[W]) {
  if constexpr (W == 8) {
    if constexpr (O == ld_order::NC) {
      asm volatile("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                   : "l"(p));
    } else if constexpr (O == ld_order::RELAXED) {
      asm volatile("ld.relaxed.gpu.global.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                   : "l"(p) : "memory");
    } else {
      asm volatile("ld.acquire.gpu.global.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                   : "l"(p) : "memory");
    }
  } else if constexpr (W == 4) {
    if constexpr (O == ld_order::NC) {
      asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(p));
    } else if constexpr (O == ld_order::RELAXED) {
      asm volatile("ld.relaxed.gpu.global.v4.u32 {%0,%1,%2,%3}, [%4];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(p) : "memory");
    } else {
      asm volatile("ld.acquire.gpu.global.v4.u32 {%0,%1,%2,%3}, [%4];"
                   : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(p) : "memory");
    }
  } else if constexpr (W == 2) {
    if constexpr (O == ld_order::NC) {
      asm volatile("ld.global.nc.v2.u32 {%0,%1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(p));
    } else if constexpr (O == ld_order::RELAXED) {
      asm volatile("ld.relaxed.gpu.global.v2.u32 {%0,%1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(p) : "memory");
    } else {
      asm volatile("ld.acquire.gpu.global.v2.u32 {%0,%1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(p) : "memory");
    }
  } else {
    if constexpr (O == ld_order::NC) {
      asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(w[0]) : "l"(p));
    } else if constexpr (O == ld_order::RELAXED) {
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(w[0]) : "l"(p) : "memory");
    } else {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(w[0]) : "l"(p) : "memory");
    }
  }
}

template <int W, st_order O>
MT_DEV void store_words(uint32_t* p, const uint32_t (&w)[W]) {
  if constexpr (W == 8) {
    if constexpr (O == st_order::WEAK) {
      asm volatile("st.global.v8.u32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                   :: "l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]) : "memory");
    } else {
      asm volatile("st.release.gpu.global.v8.u32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                   :: "l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]) : "memory");
    }
  } else if constexpr (W == 4) {
    if constexpr (O == st_order::WEAK) {
      asm volatile("st.global.v4.u32 [%0], {%1,%2,%3,%4};" :: "l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]) : "memory");
    } else {
      asm volatile("st.release.gpu.global.v4.u32 [%0], {%1,%2,%3,%4};" :: "l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]) : "memory");
    }
  } else if constexpr (W == 2) {
    if constexpr (O == st_order::WEAK) {
      asm volatile("st.global.v2.u32 [%0], {%1,%2};" :: "l"(p), "r"(w[0]), "r"(w[1]) : "memory");
    } else {
      asm volatile("st.release.gpu.global.v2.u32 [%0], {%1,%2};" :: "l"(p), "r"(w[0]), "r"(w[1]) : "memory");
    }
  } else {
    if constexpr (O == st_order::WEAK) {
      asm volatile("st.global.u32 [%0], %1;" :: "l"(p), "r"(w[0]) : "memory");
    } else {
      asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(w[0]) : "memory");
    }
  }
}

MT_DEV uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
MT_DEV uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
MT_DEV void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
MT_DEV void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
MT_DEV uint32_t atom_or_acquire(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acquire.gpu.global.or.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
MT_DEV uint32_t atom_and_release(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.release.gpu.global.and.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

template <ld_order O>
MT_DEV uint32_t ld_word(const uint32_t* p) {
  uint32_t v[1];
  load_words<1, O>(p, v);
  return v[0];
}

// Select element i (runtime) of a small register array without local memory.
template <int N>
MT_DEV uint32_t reg_select(const uint32_t (&a)[N], uint32_t i) {
  uint32_t v = a[0];
#pragma unroll
  for (int k = 1; k < N; ++k) v = (i == (uint32_t)k) ? a[k] : v;
  return v;
}
template <int N>
MT_DEV void reg_assign(uint32_t (&a)[N], uint32_t i, uint32_t v) {
#pragma unroll
  for (int k = 0; k < N; ++k) a[k] = (i == (uint32_t)k) ? v : a[k];
}

}  // namespace mtb
