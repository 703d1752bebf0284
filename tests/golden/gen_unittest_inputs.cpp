// Writes the seeded inputs of IndexinGPU's masstree unit test
// (test/unittest_masstree.cu:82-124, testing_input::make_input) for one shape,
// restated here: std::mt19937 seeded with 0, std::uniform_int_distribution for
// key and value lengths, slice s of key i of length L = (i >> (L-1-s)) + 1) * 2 + s
// where the shift count is taken modulo 32 (what the reference's
// `1u << (key_length - 1 - s)` evaluates to on x86-64 for L > 32),
// keys_not_exist = every slice + 1, values = i + 1, values2 = i + 7.
// Output (raw little-endian u32, in order): keys[n*maxK], lengths[n],
// values[n*maxV], value_lengths[n], values2[n*maxV], keys_not_exist[n*maxK],
// then the two permutations the ConcurrentMix test draws
// (test/unittest_masstree.cu:185-190 and :591-594): std::shuffle of 0..n-1 and
// of 0..10*(n/4)-1, each with a fresh std::mt19937 seeded with 0.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s n minK maxK minV maxV out.bin\n", argv[0]);
    return 2;
  }
  const uint32_t n = std::strtoul(argv[1], nullptr, 10);
  const uint32_t minK = std::strtoul(argv[2], nullptr, 10), maxK = std::strtoul(argv[3], nullptr, 10);
  const uint32_t minV = std::strtoul(argv[4], nullptr, 10), maxV = std::strtoul(argv[5], nullptr, 10);
  std::vector<uint32_t> keys((size_t)n * maxK, 0), lengths(n), values((size_t)n * maxV, 0), vlens(n),
      values2((size_t)n * maxV, 0), keys_ne((size_t)n * maxK, 0);
  std::mt19937 rng(0);
  std::uniform_int_distribution<uint32_t> kd(minK, maxK);
  std::uniform_int_distribution<uint32_t> vd(minV, maxV);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t kl = kd(rng);
    const uint32_t vl = vd(rng);
    for (uint32_t s = 0; s < kl; ++s) {
      const uint32_t factor = 1u << ((kl - 1u - s) & 31u);
      const uint32_t slice = (i / factor + 1u) * 2u + s;
      keys[(size_t)i * maxK + s] = slice;
      keys_ne[(size_t)i * maxK + s] = slice + 1u;
    }
    for (uint32_t s = 0; s < vl; ++s) {
      values[(size_t)i * maxV + s] = i + 1u;
      values2[(size_t)i * maxV + s] = i + 7u;
    }
    lengths[i] = kl;
    vlens[i] = vl;
  }
  std::vector<uint32_t> order(n), mix_order(10u * (n / 4u));
  std::iota(order.begin(), order.end(), 0u);
  std::iota(mix_order.begin(), mix_order.end(), 0u);
  {
    std::mt19937 r(0);
    std::shuffle(order.begin(), order.end(), r);
  }
  {
    std::mt19937 r(0);
    std::shuffle(mix_order.begin(), mix_order.end(), r);
  }
  FILE* f = std::fopen(argv[6], "wb");
  if (!f) return 1;
  std::fwrite(keys.data(), 4, keys.size(), f);
  std::fwrite(lengths.data(), 4, lengths.size(), f);
  std::fwrite(values.data(), 4, values.size(), f);
  std::fwrite(vlens.data(), 4, vlens.size(), f);
  std::fwrite(values2.data(), 4, values2.size(), f);
  std::fwrite(keys_ne.data(), 4, keys_ne.size(), f);
  std::fwrite(order.data(), 4, order.size(), f);
  std::fwrite(mix_order.data(), 4, mix_order.size(), f);
  std::fclose(f);
  return 0;
}
