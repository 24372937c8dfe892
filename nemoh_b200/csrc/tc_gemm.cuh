// Tensor-core trailing update of the FP32 LU (tcgen05, sm_100a).
//
// Step k of the blocked LU updates A22 -= L21 * U12 with complex FP32
// operands and a rank-32 inner dimension. On the tensor cores the complex
// product is embedded as one real GEMM,
//     [Re C; Im C] = [[Ar, -Ai], [Ai, Ar]] * [Br; Bi]        (K' = 64),
// and each operand is split into two BF16 terms x = hi + lo, keeping
// hi*hi + hi*lo + lo*hi:  A'' = [A_hi, A_hi, A_lo], B'' = [B_hi; B_lo; B_hi]
// (K'' = 192), which gives ~16-bit operands with FP32 accumulation -- ample
// for a factorization that only preconditions FP64 iterative refinement.
//
// A prep kernel writes A'' and B'' as ready-made shared-memory images
// (K-major, no swizzle, 8x8 core matrices of 128 bytes), so each CTA moves its
// operands with two bulk async copies (cp.async.bulk, no tensor map). One CTA
// computes a 64-complex-row x 128-column tile: one thread issues 12
// tcgen05.mma (M=128, N=128, K=16, BF16 -> FP32 in TMEM), the accumulator is
// read back with tcgen05.ld, staged in shared memory as complex values and
// subtracted from A22 with coalesced read-modify-writes.
// Every wait on an mbarrier is bounded; on timeout the kernel raises a status
// code, releases its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "linalg.cuh"

namespace nb200 {

constexpr int TC_ROWS = 64;                     // complex rows per tile (128 real rows)
constexpr int TC_COLS = 128;                    // columns per tile (MMA N); 2 CTAs per SM
constexpr int TC_K = 192;                       // K'' = 3 * 2 * LU_NB
constexpr int TC_SBO = (TC_K / 8) * 128;        // bytes between 8-row core-matrix groups
constexpr int TC_A_BYTES = 128 * TC_K * 2;      // 48 KB
constexpr int TC_B_BYTES = TC_COLS * TC_K * 2;  // 48 KB
constexpr int TC_SMEM = TC_A_BYTES + TC_B_BYTES + 64;
constexpr int ST_TC_TIMEOUT = 30;

struct TcWork {
  unsigned char* a = nullptr;   // A'' tiles, nsys x ceil(n/64) x 48 KB
  unsigned char* b = nullptr;   // B'' tiles, nsys x ceil(n/128) x 48 KB
  int cap_sys = 0, cap_n = 0;
  size_t total = 0;
  size_t bytes() const { return total; }
  void release() {
    cudaFree(a);
    cudaFree(b);
    a = b = nullptr;
    cap_sys = cap_n = 0;
    total = 0;
  }
  cudaError_t ensure(int nsys, int n) {
    if (nsys <= cap_sys && n <= cap_n) return cudaSuccess;
    release();
    const size_t ta = (size_t)(n + TC_ROWS - 1) / TC_ROWS, tb = (size_t)(n + TC_COLS - 1) / TC_COLS;
    cudaError_t e;
    if ((e = cudaMalloc(&a, nsys * ta * TC_A_BYTES))) return e;
    if ((e = cudaMalloc(&b, nsys * tb * TC_B_BYTES))) return e;
    cap_sys = nsys;
    cap_n = n;
    total = nsys * (ta * TC_A_BYTES + tb * TC_B_BYTES);
    return cudaSuccess;
  }
};

inline size_t tc_bytes_per_system(size_t n) {
  return ((n + TC_ROWS - 1) / TC_ROWS) * TC_A_BYTES + ((n + TC_COLS - 1) / TC_COLS) * TC_B_BYTES;
}

// byte offset of element (row, kk) in a K-major no-swizzle operand image
__device__ __forceinline__ int tc_off(int row, int kk) {
  return (row & 7) * 16 + (row >> 3) * TC_SBO + (kk >> 3) * 128 + (kk & 7) * 2;
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Build A'' (from L21) and B'' (from U12) for step k; also store the factored
// diagonal block parked by lu_panel_kernel. grid.z = system.
__global__ void tc_prep_kernel(BatchT<float2> b, int k, unsigned char* __restrict__ abuf,
                               unsigned char* __restrict__ bbuf, long long a_sys, long long b_sys) {
  const int n = b.n, nb = LU_NB, r0 = k + nb, rest = n - r0;
  float2* A = b.base + blockIdx.z * b.stride;
  const int ta = (rest + TC_ROWS - 1) / TC_ROWS, tb = (rest + TC_COLS - 1) / TC_COLS;
  unsigned char* ab = abuf + blockIdx.z * a_sys;
  unsigned char* bb = bbuf + blockIdx.z * b_sys;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  if (blockIdx.x == 0) {
    const float2* D = b.diag + (long long)blockIdx.z * LU_NB * LU_NB;
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) A[(k + q % nb) + (long long)n * (k + q / nb)] = D[q];
  }
  // A'': one complex element L21(r, j) -> 12 BF16 values
  const long long na = (long long)ta * TC_ROWS * nb;
  for (long long q = tid; q < na; q += nth) {
    const int rr = (int)(q % (ta * TC_ROWS)), j = (int)(q / (ta * TC_ROWS));
    const int t = rr / TC_ROWS, row = rr % TC_ROWS;
    float2 v = make_float2(0.f, 0.f);
    if (rr < rest) v = A[(r0 + rr) + (long long)n * (k + j)];
    __nv_bfloat16 rh, rl, ih, il, nih, nil;
    split_bf16(v.x, rh, rl);
    split_bf16(v.y, ih, il);
    nih = __hneg(ih);
    nil = __hneg(il);
    unsigned char* tile = ab + (long long)t * TC_A_BYTES;
    // real-part row: [Ar, -Ai]; imaginary-part row (row + 64): [Ai, Ar]
    const int re = row, im = row + TC_ROWS;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const bool lo = (s == 2);
      const int kb = 64 * s;
      *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(re, kb + j)) = lo ? rl : rh;
      *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(re, kb + 32 + j)) = lo ? nil : nih;
      *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(im, kb + j)) = lo ? il : ih;
      *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(im, kb + 32 + j)) = lo ? rl : rh;
    }
  }
  // B'': one complex element U12(j, c) -> 6 BF16 values in column c's K vector
  const long long nbv = (long long)tb * TC_COLS * nb;
  for (long long q = tid; q < nbv; q += nth) {
    const int j = (int)(q % nb), cc = (int)(q / nb);
    const int t = cc / TC_COLS, col = cc % TC_COLS;
    float2 v = make_float2(0.f, 0.f);
    if (cc < rest) v = A[(k + j) + (long long)n * (r0 + cc)];
    __nv_bfloat16 rh, rl, ih, il;
    split_bf16(v.x, rh, rl);
    split_bf16(v.y, ih, il);
    unsigned char* tile = bb + (long long)t * TC_B_BYTES;
    // [B_hi; B_lo; B_hi] with B' = [Br; Bi]
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, j)) = rh;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, 32 + j)) = ih;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, 64 + j)) = rl;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, 96 + j)) = il;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, 128 + j)) = rh;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc_off(col, 160 + j)) = ih;
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: about 2^22 polls with a short sleep (well under a second)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (mbar_test(bar, parity)) return true;
    __nanosleep(32);
  }
  return false;
}

// K-major, no-swizzle UMMA shared-memory descriptor (sm_100 version 1)
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for sm_100
  return d;                 // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: BF16 x BF16 -> F32, K-major A and B, M=128, N=256
__host__ __device__ constexpr uint32_t tc_idesc() {
  return (1u << 4)                    // D format F32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((uint32_t)(TC_COLS >> 3) << 17)
         | ((uint32_t)(128 >> 4) << 24);
}

__global__ void __launch_bounds__(128, 2) tc_update_kernel(BatchT<float2> b, int k, const unsigned char* __restrict__ abuf,
                                                           const unsigned char* __restrict__ bbuf, long long a_sys,
                                                           long long b_sys, int* status) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + TC_A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TC_A_BYTES + TC_B_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  const int n = b.n, r0 = k + LU_NB, rest = n - r0;
  const int tcol = blockIdx.x, trow = blockIdx.y;
  const int warp = threadIdx.x >> 5;
  const uint32_t bar_load = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);

  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_load));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mma));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (threadIdx.x == 0) {
    const unsigned char* ga = abuf + blockIdx.z * a_sys + (long long)trow * TC_A_BYTES;
    const unsigned char* gb = bbuf + blockIdx.z * b_sys + (long long)tcol * TC_B_BYTES;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_load),
                 "r"(TC_A_BYTES + TC_B_BYTES)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(sA)),
                 "l"(ga), "r"(TC_A_BYTES), "r"(bar_load)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(sB)),
                 "l"(gb), "r"(TC_B_BYTES), "r"(bar_load)
                 : "memory");
    ok = mbar_wait(bar_load, 0);
    if (ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t idesc = tc_idesc();
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int kk = 0; kk < TC_K / 16; ++kk) {
        const uint64_t da = umma_desc(a0 + kk * 256, 128, TC_SBO);
        const uint64_t db = umma_desc(b0 + kk * 256, 128, TC_SBO);
        const uint32_t acc = kk > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_mma)
                   : "memory");
      ok = mbar_wait(bar_mma, 0);
    } else {
      mbar_wait(bar_load, 0);   // give copies still in flight a second bounded chance to land
    }
    if (!ok) atomicCAS(status, 0, ST_TC_TIMEOUT);
  }
  // broadcast the outcome of thread 0's waits
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
  __syncthreads();
  ok = s_ok != 0;
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // TMEM -> registers -> shared memory, real and imaginary parts as separate
    // [col][row] float planes (reusing the operand area; conflict-free stores)
    float* sre = reinterpret_cast<float*>(smem);
    float* sim = sre + TC_COLS * TC_ROWS;
    const int trow_l = warp * 32 + (threadIdx.x & 31);  // accumulator row of this thread
    float* plane = trow_l >= TC_ROWS ? sim : sre;
    const int crow = trow_l & (TC_ROWS - 1);
    __syncthreads();
#pragma unroll 1
    for (int chunk = 0; chunk < TC_COLS / 32; ++chunk) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(chunk * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) plane[(chunk * 32 + j) * TC_ROWS + crow] = __uint_as_float(v[j]);
    }
    __syncthreads();
    // read-modify-write of the 64 x 128 tile of A22: warp w takes columns
    // w, w+4, ...; lane l takes rows 2l, 2l+1 (one 16-byte access when the
    // order n is even, so that every column starts 16-byte aligned). Sixteen
    // columns' loads are issued before any is used, to keep memory busy.
    float2* A = b.base + blockIdx.z * b.stride;
    const int lane = threadIdx.x & 31;
    const int gr = trow * TC_ROWS + 2 * lane;
    const int ncol = min(TC_COLS, rest - tcol * TC_COLS);
    const bool pair = (gr + 1 < rest) && ((n & 1) == 0);
    constexpr int UNR = 16;
    for (int c0 = warp; c0 < ncol; c0 += 4 * UNR) {
      float4 cur[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int c = c0 + 4 * u;
        if (c < ncol && gr < rest) {
          float2* p = A + (r0 + gr) + (long long)n * (r0 + tcol * TC_COLS + c);
          if (pair) cur[u] = *reinterpret_cast<const float4*>(p);
          else cur[u] = make_float4(p[0].x, p[0].y, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int c = c0 + 4 * u;
        if (c < ncol && gr < rest) {
          float2* p = A + (r0 + gr) + (long long)n * (r0 + tcol * TC_COLS + c);
          const int q = c * TC_ROWS + 2 * lane;
          float4 o = cur[u];
          o.x -= sre[q];
          o.y -= sim[q];
          if (pair) {
            o.z -= sre[q + 1];
            o.w -= sim[q + 1];
            *reinterpret_cast<float4*>(p) = o;
          } else {
            p[0] = make_float2(o.x, o.y);
            if (gr + 1 < rest) {
              float2 t = p[1];
              t.x -= sre[q + 1];
              t.y -= sim[q + 1];
              p[1] = t;
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS));
}

inline bool tc_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("NEMOH_B200_TC");
    on = (e && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}

// Trailing update of step k on the tensor cores. Returns false when the
// SIMT update should be used instead (disabled, or no trailing matrix).
inline bool tc_update(TcWork& w, BatchT<float2> b, int k, int nb, int nsys, cudaStream_t st, long long& launches,
                      int* status) {
  const int rest = b.n - k - nb;
  if (!tc_enabled() || rest <= 0 || nb != LU_NB || !w.a) return false;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(tc_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM) != cudaSuccess)
      return false;
    attr = true;
  }
  const long long a_sys = (long long)((w.cap_n + TC_ROWS - 1) / TC_ROWS) * TC_A_BYTES;
  const long long b_sys = (long long)((w.cap_n + TC_COLS - 1) / TC_COLS) * TC_B_BYTES;
  const int ta = (rest + TC_ROWS - 1) / TC_ROWS, tb = (rest + TC_COLS - 1) / TC_COLS;
  tc_prep_kernel<<<dim3(std::max(1, std::min(64, ta * 2)), 1, nsys), 256, 0, st>>>(b, k, w.a, w.b, a_sys, b_sys);
  ++launches;
  tc_update_kernel<<<dim3(tb, ta, nsys), 128, TC_SMEM, st>>>(b, k, w.a, w.b, a_sys, b_sys, status);
  ++launches;
  return true;
}

}  // namespace nb200
