// Compiles (and, on a GPU, runs) a small program against the C++ host mirror
// include/mt/gpu_masstree.hpp and libmt_b200.so: insert, find, validate,
// written the way the reference's host API is called, plus a mixed batch from
// host buffers.
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
  // Host buffers: erase every second key and find all keys through the
  // host-buffer entry point (two chunks).
  std::vector<uint8_t> types(n);
  std::vector<uint32_t> hv(n * maxV, 0), hvl(n, 0);
  for (uint32_t i = 0; i < n; ++i) types[i] = (i % 2) ? (uint8_t)request_type_erase : (uint8_t)request_type_find;
  std::vector<uint8_t> res(n, 0);
  tree.mixed_batch_host(reinterpret_cast<const request_type*>(types.data()), keys.data(), maxK, klens.data(),
                        hv.data(), maxV, hvl.data(), reinterpret_cast<bool*>(res.data()), n, 0, 600);
  cudaStreamSynchronize(0);
  for (uint32_t i = 0; i < n; ++i) {
    if (i % 2) bad += res[i] != 1;          // erased
    else bad += hvl[i] != vlens[i];         // found with its value length
  }
  std::string report;
  bad += !tree.validate(&report);
  std::printf("host api check: %s, %d mismatches\n", report.c_str(), bad);
  return bad ? 1 : 0;
}
