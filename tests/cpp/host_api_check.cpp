// Compiles (and, on a GPU, runs) a small program against the C++ host mirror
// include/mt/gpu_masstree.hpp and libmt_b200.so: insert, find, mixed_batch,
// scan, validate, written the way the reference's host API is called.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "mt/gpu_masstree.hpp"

int main() {
  using namespace GpuMasstreeB200;
  const uint32_t n = 1000, maxK = 3, maxV = 2;
  std::vector<uint32_t> keys(n * maxK), klens(n), vals(n * maxV), vlens(n);
  for (uint32_t i = 0; i < n; ++i) {
    klens[i] = 1 + i % 3;
    for (uint32_t s = 0; s < klens[i]; ++s) keys[i * maxK + s] = i * 7 + s;
    vlens[i] = 1 + i % 2;
    for (uint32_t s = 0; s < vlens[i]; ++s) vals[i * maxV + s] = i + 100 * s;
  }
  uint32_t *dk, *dkl, *dv, *dvl, *ov, *ovl;
  cudaMalloc(&dk, keys.size() * 4); cudaMalloc(&dkl, n * 4); cudaMalloc(&dv, vals.size() * 4);
  cudaMalloc(&dvl, n * 4); cudaMalloc(&ov, vals.size() * 4); cudaMalloc(&ovl, n * 4);
  cudaMemcpy(dk, keys.data(), keys.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dkl, klens.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dv, vals.data(), vals.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dvl, vlens.data(), n * 4, cudaMemcpyHostToDevice);
  gpu_masstree tree(0.01f);
  tree.insert(dk, maxK, dkl, dv, maxV, dvl, n);
  tree.find(dk, maxK, dkl, ov, maxV, ovl, n);
  std::vector<uint32_t> got(n);
  cudaMemcpy(got.data(), ovl, n * 4, cudaMemcpyDeviceToHost);
  int bad = tree.last_error() != MT_OK;
  for (uint32_t i = 0; i < n; ++i) bad += got[i] != vlens[i];
  std::string report;
  bad += !tree.validate(&report);
  std::printf("host api check: %s, %d mismatches\n", report.c_str(), bad);
  return bad ? 1 : 0;
}
