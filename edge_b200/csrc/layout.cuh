// Conversion between the reference DOF layout of the C ABI, [nEl][rows][B][R] (runs fastest,
// src/data/Internal.hpp:559-568), and the device-resident row layout [nEl][rows][R][G] (modes
// fastest, rows padded to G elements; see kernels.cuh). One CTA per (element, quantity row)
// stages the B x R block in shared memory so both sides are read and written contiguously.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace edge_b200 {

constexpr int kLayoutThreads = 256;
constexpr int kLayoutMaxBlock = 56 * 32;  // B * R of the largest configuration (order 6, 32 runs)

template <typename T>
__global__ void __launch_bounds__(kLayoutThreads) kToRows(const T *__restrict__ ref, T *__restrict__ rows,
                                                          int64_t nBlocks, int B, int R, int G) {
  __shared__ T tile[kLayoutMaxBlock];
  for (int64_t blk = blockIdx.x; blk < nBlocks; blk += gridDim.x) {
    const T *src = ref + blk * int64_t(B) * R;
    for (int i = threadIdx.x; i < B * R; i += blockDim.x) tile[i] = src[i];  // [B][R]
    __syncthreads();
    T *dst = rows + blk * int64_t(R) * G;
    for (int i = threadIdx.x; i < R * G; i += blockDim.x) {
      const int r = i / G, n = i % G;
      dst[i] = n < B ? tile[n * R + r] : T(0);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(kLayoutThreads) kFromRows(const T *__restrict__ rows, T *__restrict__ ref,
                                                            int64_t nBlocks, int B, int R, int G) {
  __shared__ T tile[kLayoutMaxBlock];
  for (int64_t blk = blockIdx.x; blk < nBlocks; blk += gridDim.x) {
    const T *src = rows + blk * int64_t(R) * G;
    for (int i = threadIdx.x; i < R * G; i += blockDim.x) {
      const int r = i / G, n = i % G;
      if (n < B) tile[n * R + r] = src[i];
    }
    __syncthreads();
    T *dst = ref + blk * int64_t(B) * R;
    for (int i = threadIdx.x; i < B * R; i += blockDim.x) dst[i] = tile[i];
    __syncthreads();
  }
}

// launches one of the conversions for nBlocks (element, row) blocks; precision 32 or 64
inline cudaError_t convertLayout(bool toRows, int precision, const void *in, void *out, int64_t nBlocks, int B,
                                 int R, int G, cudaStream_t s) {
  if (nBlocks <= 0) return cudaSuccess;
  if (B * R > kLayoutMaxBlock) return cudaErrorInvalidValue;
  const int grid = (int)(nBlocks < 65536 ? nBlocks : 65536);
  if (precision == 64) {
    if (toRows)
      kToRows<double><<<grid, kLayoutThreads, 0, s>>>((const double *)in, (double *)out, nBlocks, B, R, G);
    else
      kFromRows<double><<<grid, kLayoutThreads, 0, s>>>((const double *)in, (double *)out, nBlocks, B, R, G);
  } else {
    if (toRows)
      kToRows<float><<<grid, kLayoutThreads, 0, s>>>((const float *)in, (float *)out, nBlocks, B, R, G);
    else
      kFromRows<float><<<grid, kLayoutThreads, 0, s>>>((const float *)in, (float *)out, nBlocks, B, R, G);
  }
  return cudaGetLastError();
}

// padded row lengths of the device-resident layout (16-byte rows)
inline int rowPad(int n, int precision) {
  const int w = precision == 64 ? 2 : 4;
  return ((n + w - 1) / w) * w;
}

}  // namespace edge_b200
