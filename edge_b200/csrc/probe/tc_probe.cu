// Measurement probe for the tensor-core question of the element update: how fast does one
// tcgen05.mma (kind::tf32 or kind::f16 with bf16 operands, operands in shared memory, accumulator
// in tensor memory) run at the small shapes the DG products of the local kernel would have (M = 128
// rows of (quantity, element, run), N = 16..128 output modes, K = 8 (tf32) or 16 (bf16) per
// instruction), with one or two issuing CTAs per SM, and does its result match the FP32 product.
// Built into its own library (libedge_b200_probe.so): it is not part of the element update, only
// the evidence for keeping those products on the FP32 pipe.
//
// Operands use the K-major SWIZZLE_NONE canonical layout of the shared-memory matrix descriptor:
// core matrices of 8 rows x 16 bytes (4 tf32 or 8 bf16) stored contiguously (128 bytes); the 8-row
// groups of one 16-byte K chunk follow each other (stride-dimension offset 128 bytes) and the K
// chunks follow the row groups (leading-dimension offset rows / 8 * 128 bytes). One instruction
// reads two K chunks (32 bytes of every row) in both kinds.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kThreads = 128;      // four warps: the 128 accumulator lanes, one warp per 32
constexpr int kMaxRows = 128;      // M (A rows) and N (B rows) at most
constexpr int kRowBytes = 128;     // staged K per row: 32 tf32 or 64 bf16
constexpr long long kWaitCycles = 4000000000LL;  // about two seconds at the boost clock
// dynamic shared memory per CTA: the two operand tiles plus padding that sets the CTAs per SM (one
// or two); the host admits two only where their tensor-memory allocations fit side by side, so no
// allocation waits on another CTA
constexpr int kSmemOne = 120 * 1024, kSmemTwo = 96 * 1024;

__device__ __forceinline__ uint32_t smemAddr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row r, k) in the canonical K-major layout of a tile with `rows` rows and
// `eb` bytes per element
__host__ __device__ __forceinline__ uint32_t canonOffset(int r, int k, int rows, int eb) {
  const int per = 16 / eb;
  return (uint32_t)((k / per) * (rows / 8) * 128 + (r / 8) * 128 + (r % 8) * 16 + (k % per) * eb);
}

__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
  return d;
}

// tensor-memory columns one CTA allocates: acc accumulators of n columns, each on a 32-column
// boundary, rounded up to a power of two (at least 32)
__host__ __device__ __forceinline__ uint32_t accStride(int n) { return ((uint32_t)n + 31) / 32 * 32; }
__host__ __device__ __forceinline__ uint32_t tmemCols(int n, int acc) {
  uint32_t cols = 32;
  while (cols < accStride(n) * (uint32_t)acc) cols <<= 1;
  return cols;
}

// instruction descriptor: D f32, A and B tf32 (format 2) or bf16 (format 1; same type for both),
// both K-major, N / 8 and M / 16
__host__ __device__ constexpr uint32_t instrDesc(int m, int n, bool bf16) {
  return (1u << 4) | ((bf16 ? 1u : 2u) << 7) | ((bf16 ? 1u : 2u) << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

template <bool BF16>
__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                    uint32_t accumulate) {
  if (BF16)
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// element i of a staged operand, rounded to the instruction's input type when that is bf16 (tf32
// reads the FP32 bits and ignores the low 13)
template <bool BF16>
__device__ __forceinline__ void stage(char *tile, int r, int c, int rows, float v) {
  if (BF16)
    *reinterpret_cast<__nv_bfloat16 *>(tile + canonOffset(r, c, rows, 2)) = __float2bfloat16_rn(v);
  else
    *reinterpret_cast<float *>(tile + canonOffset(r, c, rows, 4)) = v;
}

__device__ __forceinline__ bool waitParity(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (clock64() - t0 < kWaitCycles) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One CTA per block: A [m][k] and B [n][k] (row-major in global memory, k = KB x the instruction's
// K) staged into the canonical layout; `iters` passes, each issuing for every K block one instruction into
// each of ACC independent accumulators [m][n] in tensor memory (ACC = 1: every instruction waits
// for the previous one's sum; more: their latencies overlap, as the row tiles of an element group
// would). Descriptors are computed once and the issue loop is unrolled, so the single issuing
// thread adds little beyond the instructions themselves. Accumulator 0 is written back to D (block
// 0 only) so the host can check it against the FP32 product. status[blockIdx.x]: 0 ok, 1 the
// completion wait gave up.
template <int ACC, int KB, bool BF16>
__global__ void __launch_bounds__(kThreads, 1)
    kTcProbe(const float *A, const float *B, float *D, int m, int n, int iters, int *status) {
  constexpr int k = (BF16 ? 16 : 8) * KB;
  extern __shared__ __align__(128) char dyn[];
  char *sA = dyn, *sB = dyn + kMaxRows * kRowBytes;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmemBase;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < m * k; i += kThreads) {
    stage<BF16>(sA, i / k, i % k, m, A[i]);
  }
  for (int i = tid; i < n * k; i += kThreads) {
    stage<BF16>(sB, i / k, i % k, n, B[i]);
  }
  const uint32_t barAddr = smemAddr(&bar);
  const uint32_t stride = accStride(n), cols = tmemCols(n, ACC);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barAddr) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemAddr(&tmemBase)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // operands written by threads become visible to the tensor core's (async) proxy
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmemBase;
  if (tid == 0) {
    const uint32_t idesc = instrDesc(m, n, BF16);
    const uint32_t aBase = smemAddr(sA), bBase = smemAddr(sB);
    const uint32_t aLbo = (uint32_t)(m / 8) * 128, bLbo = (uint32_t)(n / 8) * 128;
    uint64_t ad[KB], bd[KB];
    uint32_t dc[ACC];
#pragma unroll
    for (int kb = 0; kb < KB; kb++) {
      ad[kb] = smemDesc(aBase + 2 * kb * aLbo, aLbo, 128);
      bd[kb] = smemDesc(bBase + 2 * kb * bLbo, bLbo, 128);
    }
#pragma unroll
    for (int a = 0; a < ACC; a++) dc[a] = tmem + (uint32_t)a * stride;
    for (int it = 0; it < iters; it++) {
#pragma unroll
      for (int kb = 0; kb < KB; kb++)
#pragma unroll
        for (int a = 0; a < ACC; a++) mma<BF16>(dc[a], ad[kb], bd[kb], idesc, (it > 0 || kb > 0) ? 1u : 0u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(barAddr)
                 : "memory");
  }
  bool ok = waitParity(barAddr, 0);
  if (!ok) ok = waitParity(barAddr, 0);  // second bounded wait for the work in flight before freeing
  if (!ok && tid == 0) status[blockIdx.x] = 1;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (ok && blockIdx.x == 0 && D) {
    // warp w reads accumulator lanes 32 w .. 32 w + 31 (rows of D), 8 columns per load
    const int row = warp * 32 + (tid & 31);
    for (int c0 = 0; c0 < n; c0 += 8) {
      uint32_t v[8];
      const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (row < m)
        for (int j = 0; j < 8 && c0 + j < n; j++) D[row * n + c0 + j] = __uint_as_float(v[j]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(cols) : "memory");
}

}  // namespace

extern "C" {

// Runs the probe: `blocks` CTAs (per_sm of them per SM: 1 or 2), each `iters` x KB x acc MMAs of
// shape m x n x K (kind 0: tf32, K 8; kind 1: bf16, K 16) on its own operand copies (A [m][k],
// B [n][k] FP32 device arrays, rounded to bf16 when staged for kind 1; D [m][n] device array or
// NULL: accumulator 0) into acc (1 or 3) independent accumulators. m = 128, n a multiple of 16 in
// [16, 128], k = K or 4 K (KB = 1 or 4); two CTAs per SM only where both tensor-memory allocations
// fit (2 x columns <= 512). Returns 0, -1 for invalid arguments, -3 for a CUDA error; *ms receives
// the kernel time (CUDA events), status[blocks] the per-CTA completion flags (device array).
int edge_b200_probe_tc(const float *A, const float *B, float *D, int m, int n, int k, int iters, int acc,
                       int blocks, int kind, int per_sm, int *status, float *ms) {
  const int kInstr = kind == 1 ? 16 : 8;
  if (m != 128 || n < 16 || n > kMaxRows || n % 16 || (kind != 0 && kind != 1) || (k != kInstr && k != 4 * kInstr) ||
      iters < 1 || blocks < 1 || (acc != 1 && acc != 3) || (per_sm != 1 && per_sm != 2) ||
      (uint32_t)per_sm * tmemCols(n, acc) > 512 || !A || !B || !status || !ms)
    return -1;
  const bool kb4 = k == 4 * kInstr;
  void (*kern)(const float *, const float *, float *, int, int, int, int *);
  if (kind == 0)
    kern = acc == 1 ? (kb4 ? kTcProbe<1, 4, false> : kTcProbe<1, 1, false>)
                    : (kb4 ? kTcProbe<3, 4, false> : kTcProbe<3, 1, false>);
  else
    kern = acc == 1 ? (kb4 ? kTcProbe<1, 4, true> : kTcProbe<1, 1, true>)
                    : (kb4 ? kTcProbe<3, 4, true> : kTcProbe<3, 1, true>);
  const int smem = per_sm == 1 ? kSmemOne : kSmemTwo;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -3;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -3;
  cudaEventRecord(e0);
  kern<<<blocks, kThreads, smem>>>(A, B, D, m, n, iters, status);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaGetLastError();
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return err == cudaSuccess ? 0 : -3;
}

}  // extern "C"
