// Tensor-core trailing update of the mixed-precision LU (tcgen05, sm_100a).
//
// The FP32 LU (mixed.cuh) factors 128-column panels with 32-column steps and
// then updates the trailing matrix once per panel:
//     A22 <- A22 - L21 * U12        (complex FP32, inner dimension K = 128).
// On the tensor cores the complex product becomes real 16-bit products with
// FP32 accumulation. A is kept as [Ar | Ai] (K' = 2K real columns) and B as two
// column blocks, [Br; -Bi] for the real parts and [Bi; Br] for the imaginary
// parts of the result (N' = 2 x 128), so that
//     [Re C | Im C] = [Ar | Ai] * [[Br, Bi], [-Bi, Br]].
// Each operand is split x = hi + lo into two BF16 terms (16 significant bits;
// FP16 terms, 22 bits, with NEMOH_B200_TC_SPLIT=f16) and the product keeps
// hi*hi + hi*lo + lo*hi (FP32 accumulation): the same hi and lo images are
// reused by three MMAs through their descriptors, so they are stored once.
//
// A prep kernel writes both operands as ready-made shared-memory images
// (K-major, no swizzle, 8x8 core matrices of 128 bytes) per tile and per
// chunk of 16 complex k. One CTA computes a 128 x 128 complex tile: thread 0
// streams the chunks through two shared-memory stages with bulk async copies
// and issues 6 tcgen05.mma (M=128, N=256, K=16) per chunk into a 256-column
// TMEM accumulator; afterwards every thread reads its row of the accumulator
// with tcgen05.ld and subtracts it from A22 with coalesced column accesses.
// Every wait on an mbarrier is bounded; on timeout the kernel raises a status
// code, waits (bounded) for its copies and MMAs in flight, releases its tensor
// memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "linalg.cuh"

namespace nb200 {

constexpr int TC_T = 128;                       // complex rows and columns per tile
constexpr int TC_KC = 16;                       // complex k per chunk
constexpr int TC_NCH = LU_OUTER / TC_KC;        // chunks per update
constexpr int TC_SBO = (2 * TC_KC / 8) * 128;   // 512 bytes between 8-row core-matrix groups
constexpr int TC_AIMG = TC_T * 2 * TC_KC * 2;   // 8 KB: one A image (hi or lo) of a chunk
constexpr int TC_BIMG = 2 * TC_T * 2 * TC_KC * 2;   // 16 KB: one B image of a chunk
constexpr int TC_STAGE = 2 * TC_AIMG + 2 * TC_BIMG;  // 48 KB: A hi, A lo, B hi, B lo
constexpr int TC_SMEM = 2 * TC_STAGE + 128;
constexpr int TC_TMEM_COLS = 2 * TC_T;          // accumulator: Re in [0,128), Im in [128,256)
constexpr int ST_TC_TIMEOUT = 30;

// Operand images of two outer updates (two sets: the update of one panel may
// be merged into the next panel's, and both panels' images are then read).
constexpr long long TC_W_BYTES = (long long)TC_NCH * 2 * TC_BIMG;   // one B tile of K = 128 (conj(W^T))
constexpr long long TC_V_BYTES = (long long)TC_NCH * 2 * TC_BIMG;   // one B tile of K = 128
constexpr long long TC_WV_BYTES = TC_W_BYTES + TC_V_BYTES;

struct TcWork {
  unsigned char* a = nullptr;   // A images: 2 sets x nsys x ceil(n/128) row tiles x TC_NCH chunks x (hi, lo)
  unsigned char* b = nullptr;   // B images: 2 sets x nsys x ceil(n/128) column tiles x TC_NCH chunks x (hi, lo)
  // per system: the B images of conj(W^T), W = inv(L11), and of V = inv(U11)
  // (the panel's block products on the tensor cores)
  unsigned char* wv = nullptr;
  size_t have_a = 0, have_b = 0, have_wv = 0;
  size_t bytes() const { return have_a + have_b + have_wv; }
  // the images of set s (0 or 1), each set half of the allocation
  TcWork set(int s) const {
    TcWork w = *this;
    w.a += s * (have_a / 2);
    w.b += s * (have_b / 2);
    return w;
  }
  void release() {
    cudaFree(a);
    cudaFree(b);
    cudaFree(wv);
    a = b = wv = nullptr;
    have_a = have_b = have_wv = 0;
  }
  cudaError_t ensure(int nsys, int n, bool headroom = false) {
    const size_t t = (size_t)(n + TC_T - 1) / TC_T;
    const size_t na = 2 * nsys * t * TC_NCH * 2 * TC_AIMG, nb = 2 * nsys * t * TC_NCH * 2 * TC_BIMG;
    cudaError_t e = grow_alloc(reinterpret_cast<void**>(&a), &have_a, na, headroom);
    if (e) return e;
    e = grow_alloc(reinterpret_cast<void**>(&wv), &have_wv, (size_t)nsys * TC_WV_BYTES, headroom);
    if (e) return e;
    return grow_alloc(reinterpret_cast<void**>(&b), &have_b, nb, headroom);
  }
};

inline size_t tc_bytes_per_system(size_t n) {
  return 2 * ((n + TC_T - 1) / TC_T) * TC_NCH * 2 * (size_t)(TC_AIMG + TC_BIMG) + TC_WV_BYTES;
}

// byte offset of the 16-byte core-matrix row (row, k-group g) in an image
__device__ __forceinline__ int tc_row_off(int row, int g) { return (row & 7) * 16 + (row >> 3) * TC_SBO + g * 128; }

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) {
  return (uint32_t)__bfloat16_as_ushort(v.x) | ((uint32_t)__bfloat16_as_ushort(v.y) << 16);
}

__device__ __forceinline__ uint32_t h2_bits(__half2 v) {
  return (uint32_t)__half_as_ushort(v.x) | ((uint32_t)__half_as_ushort(v.y) << 16);
}

// eight consecutive values -> hi terms and lo = x - hi terms, packed in k
// order (element 0 in the low half of the first word); BF16 terms, or FP16
// terms (F16: 11-bit significands, so hi + lo keeps 22 bits against 16 with
// BF16; the LU factors the dimensionless matrix D, whose entries are far
// inside FP16's range, and a lo term below FP16's normal range loses only
// what is already below 2^-24 of the largest entries)
template <bool F16>
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (F16) {
      const __half2 h2 = __floats2half2_rn(x[2 * i], x[2 * i + 1]);
      const float2 hf = __half22float2(h2);
      h[i] = h2_bits(h2);
      l[i] = h2_bits(__floats2half2_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y));
    } else {
      const __nv_bfloat162 h2 = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
      const float2 hf = __bfloat1622float2(h2);
      h[i] = bf2_bits(h2);
      l[i] = bf2_bits(__floats2bfloat162_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y));
    }
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Operand images of the outer update after the panel [k0, k0 + 128):
// L21 = A[r1:n, k0:k0+128] and U12 = A[k0:k0+128, r1:n] with r1 = k0 + 128.
// Thread per (row or column of the tile, chunk); blocks [0, na) do A, the rest B.
template <bool F16>
__global__ void __launch_bounds__(128) tc_prep_kernel(BatchT<float2> b, int k0, unsigned char* __restrict__ abuf,
                                                       unsigned char* __restrict__ bbuf, long long sys_bytes_a,
                                                       long long sys_bytes_b, int na) {
  const int n = b.order(blockIdx.z), r1 = k0 + LU_OUTER, rest = n - r1;
  if (rest <= 0) return;
  const int nt = (rest + TC_T - 1) / TC_T;
  const float2* A = b.sys(blockIdx.z);
  const bool isA = (int)blockIdx.x < na;
  const int q = (isA ? blockIdx.x : blockIdx.x - na) * blockDim.x + threadIdx.x;
  if (q >= nt * TC_T * TC_NCH) return;
  const int ch = q / (nt * TC_T), rr = q % (nt * TC_T);   // consecutive threads: consecutive rows/columns
  const int t = rr / TC_T, row = rr % TC_T;
  const int kb = k0 + ch * TC_KC;
  float re[TC_KC], im[TC_KC];
  if (isA) {
    const int r = r1 + rr;
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) {
      const float2 v = (r < n) ? A[r + (long long)n * (kb + j)] : make_float2(0.f, 0.f);
      re[j] = v.x;
      im[j] = v.y;
    }
    unsigned char* img = abuf + blockIdx.z * sys_bytes_a + ((long long)t * TC_NCH + ch) * 2 * TC_AIMG;
    uint4 h, l;
    // k-groups: 0,1 = Re(k 0..15), 2,3 = Im(k 0..15)
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      split8<F16>((g < 2 ? re : im) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_AIMG + tc_row_off(row, g)) = l;
    }
  } else {
    const int c = r1 + rr;
    const float2* col = A + (long long)n * c + kb;
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) {
      const float2 v = (c < n) ? col[j] : make_float2(0.f, 0.f);
      re[j] = v.x;
      im[j] = v.y;
    }
    float nim[TC_KC];
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) nim[j] = -im[j];
    unsigned char* img = bbuf + blockIdx.z * sys_bytes_b + ((long long)t * TC_NCH + ch) * 2 * TC_BIMG;
    uint4 h, l;
    // B row `row` (real parts of the result): [Br; -Bi]; row 128+row (imaginary parts): [Bi; Br]
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      split8<F16>((g < 2 ? re : nim) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(row, g)) = l;
      split8<F16>((g < 2 ? im : re) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(TC_T + row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(TC_T + row, g)) = l;
    }
  }
}

// Images of the panel's W = inv(L11) and V = inv(U11), K = 128, in the
// layout of tc_prep_kernel's, for the block products on the tensor cores:
// V as the B tile of L21 = A21 V, and conj(W^T) as the B tile of
// conj(U12^T) = conj(A12^T) conj(W^T), the transposed form of U12 = W A12
// (its A operand, conj(A12^T), is the first half of A12's B image, and each
// accumulator row is then one column of U12). Blocks [0, 8): W, [8, 16): V.
template <bool F16>
__global__ void __launch_bounds__(128) tc_prep_wv_kernel(BatchT<float2> b, int k0, unsigned char* __restrict__ wv) {
  const int n = b.order(blockIdx.z);
  if (k0 + LU_OUTER >= n) return;
  const float2* P = b.pinv + (long long)blockIdx.z * PINV_SCRATCH;
  constexpr int PER = TC_T * TC_NCH / 128;
  const bool isW = (int)blockIdx.x < PER;
  const int q = (isW ? blockIdx.x : blockIdx.x - PER) * 128 + threadIdx.x;   // < TC_T * TC_NCH
  const int ch = q / TC_T, row = q % TC_T, kb = ch * TC_KC;
  unsigned char* base = wv + blockIdx.z * TC_WV_BYTES;
  float re[TC_KC], im[TC_KC];
  uint4 h, l;
  if (isW) {   // B column `row` of conj(W^T): conj(W[row, kb + j])
    const float2* W = P + PINV_W_OFF;
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) {
      const float2 v = W[row + LU_OUTER * (kb + j)];
      re[j] = v.x;
      im[j] = v.y;
    }
    float nim[TC_KC];
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) nim[j] = -im[j];
    unsigned char* img = base + (long long)ch * 2 * TC_BIMG;
    // B column of Y = conj(W^T): [Re Y; -Im Y] = [Re W; Im W], [Im Y; Re Y] = [-Im W; Re W]
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      split8<F16>((g < 2 ? re : im) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(row, g)) = l;
      split8<F16>((g < 2 ? nim : re) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(TC_T + row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(TC_T + row, g)) = l;
    }
  } else {     // B column `row` of V: V[kb + j, row]
    const float2* V = P + PINV_V_OFF;
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) {
      const float2 v = V[(kb + j) + LU_OUTER * row];
      re[j] = v.x;
      im[j] = v.y;
    }
    float nim[TC_KC];
#pragma unroll
    for (int j = 0; j < TC_KC; ++j) nim[j] = -im[j];
    unsigned char* img = base + TC_W_BYTES + (long long)ch * 2 * TC_BIMG;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      split8<F16>((g < 2 ? re : nim) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(row, g)) = l;
      split8<F16>((g < 2 ? im : re) + 8 * (g & 1), h, l);
      *reinterpret_cast<uint4*>(img + tc_row_off(TC_T + row, g)) = h;
      *reinterpret_cast<uint4*>(img + TC_BIMG + tc_row_off(TC_T + row, g)) = l;
    }
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

// instruction descriptor: BF16 x BF16 (or F16 x F16: A and B always share
// the type) -> F32, K-major A and B, M=128, N=256
__host__ __device__ constexpr uint32_t tc_idesc(bool f16 = false) {
  return (1u << 4)                    // D format F32
         | (f16 ? 0u : 1u << 7)       // A format: F16 (0) or BF16 (1)
         | (f16 ? 0u : 1u << 10)      // B format: the same as A
         | ((uint32_t)((2 * TC_T) >> 3) << 17)
         | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_load_chunk(uint32_t dst, const unsigned char* ga, const unsigned char* gb,
                                              uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TC_STAGE) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(ga), "r"(2 * TC_AIMG), "r"(bar)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst + 2 * TC_AIMG),
               "l"(gb), "r"(2 * TC_BIMG), "r"(bar)
               : "memory");
}

// the same stage with the A chunk's hi and lo halves from two places (the
// first 128 rows of a B image's hi and lo terms)
__device__ __forceinline__ void tc_load_chunk_split(uint32_t dst, const unsigned char* ga_hi,
                                                    const unsigned char* ga_lo, const unsigned char* gb,
                                                    uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TC_STAGE) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(ga_hi), "r"(TC_AIMG), "r"(bar)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst + TC_AIMG),
               "l"(ga_lo), "r"(TC_AIMG), "r"(bar)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst + 2 * TC_AIMG),
               "l"(gb), "r"(2 * TC_BIMG), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

// A[r1:n, r1:n] -= L21 U12 for the panel [k0, k0+128), r1 = k0 + 128.
// grid = (column tiles, row tiles, systems), 128 threads, TC_SMEM dynamic smem.
__global__ void __launch_bounds__(128, 2) tc_update_kernel(BatchT<float2> b, int k0,
                                                           const unsigned char* __restrict__ abuf,
                                                           const unsigned char* __restrict__ bbuf,
                                                           long long sys_bytes_a, long long sys_bytes_b, int* status,
                                                           uint32_t idesc, int ti0, int tj0) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * TC_STAGE);   // full[2], empty[2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 4);
  __shared__ int s_ok;
  const int n = b.order(blockIdx.z), r1 = k0 + LU_OUTER, rest = n - r1;
  // column tiles [tj0, tj0 + gridDim.x), row tiles [ti0, ti0 + gridDim.y)
  const int tcol = blockIdx.x + tj0, trow = blockIdx.y + ti0;
  // a ragged batch's smaller systems leave the tiles beyond their order
  // (uniform per CTA, before any barrier or tensor-memory allocation)
  if (rest <= 0 || tcol * TC_T >= rest || trow * TC_T >= rest) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[2]);

  if (threadIdx.x == 0) {
    for (int i = 0; i < 4; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[i])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // while thread 0 streams the operands and issues the MMAs, every thread
  // pulls one column of this CTA's 128 x 128 result tile into L2, so that the
  // read-modify-write at the end reads from L2 instead of HBM
  {
    const int gr0 = r1 + trow * TC_T, nrows = min(TC_T, n - gr0);
    const int c = r1 + tcol * TC_T + (int)threadIdx.x;
    if (nrows > 0 && c < n) {
      const char* p = reinterpret_cast<const char*>(b.sys(blockIdx.z) + gr0 + (long long)n * c);
      for (int off = 0; off < nrows * (int)sizeof(float2); off += 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p + off));
    }
  }

  if (threadIdx.x == 0) {
    bool ok = true;
    const unsigned char* ga = abuf + blockIdx.z * sys_bytes_a + (long long)trow * TC_NCH * 2 * TC_AIMG;
    const unsigned char* gb = bbuf + blockIdx.z * sys_bytes_b + (long long)tcol * TC_NCH * 2 * TC_BIMG;
    const uint32_t s0 = smem_u32(smem);
    tc_load_chunk(s0, ga, gb, full0);
    tc_load_chunk(s0 + TC_STAGE, ga + 2 * TC_AIMG, gb + 2 * TC_BIMG, full0 + 8);
    int issued = 2;      // chunks whose loads were issued
    int committed = 0;   // chunks whose MMAs were committed
    for (int c = 0; c < TC_NCH && ok; ++c) {
      const int s = c & 1;
      const uint32_t par = (uint32_t)((c >> 1) & 1);
      ok = mbar_wait(full0 + 8 * s, par);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t st = s0 + s * TC_STAGE;
      const uint32_t ahi = st, alo = st + TC_AIMG, bhi = st + 2 * TC_AIMG, blo = bhi + TC_BIMG;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        const uint32_t o = kk * 256;
        tc_mma(tmem, umma_desc(ahi + o, 128, TC_SBO), umma_desc(bhi + o, 128, TC_SBO), (c > 0 || kk > 0) ? 1u : 0u,
               idesc);
        tc_mma(tmem, umma_desc(ahi + o, 128, TC_SBO), umma_desc(blo + o, 128, TC_SBO), 1u, idesc);
        tc_mma(tmem, umma_desc(alo + o, 128, TC_SBO), umma_desc(bhi + o, 128, TC_SBO), 1u, idesc);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(empty0 + 8 * s)
                   : "memory");
      committed = c + 1;
      // refill the stage of chunk c-1 with chunk c+1 once its MMAs are done
      if (c >= 1 && c + 1 < TC_NCH && issued == c + 1) {
        const int sp = (c - 1) & 1;
        ok = mbar_wait(empty0 + 8 * sp, (uint32_t)(((c - 1) >> 1) & 1));
        if (!ok) break;
        tc_load_chunk(s0 + sp * TC_STAGE, ga + (long long)(c + 1) * 2 * TC_AIMG, gb + (long long)(c + 1) * 2 * TC_BIMG,
                      full0 + 8 * sp);
        ++issued;
      }
    }
    if (ok) {
      // the last commit arrives when every MMA issued before it has completed
      const int c = TC_NCH - 1;
      ok = mbar_wait(empty0 + 8 * (c & 1), (uint32_t)((c >> 1) & 1));
    }
    if (!ok) {
      atomicCAS(status, 0, ST_TC_TIMEOUT);
      // give copies and MMAs still in flight a second bounded chance to finish
      for (int c = committed; c < issued; ++c) mbar_wait(full0 + 8 * (c & 1), (uint32_t)((c >> 1) & 1));
      if (committed > 0) {
        const int c = committed - 1;
        mbar_wait(empty0 + 8 * (c & 1), (uint32_t)((c >> 1) & 1));
      }
    }
    s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  if (s_ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // row `row` of the tile = TMEM lane; columns [0,128) real, [128,256) imaginary
    const int row = warp * 32 + lane;
    const int gr = r1 + trow * TC_T + row;
    float2* A = b.sys(blockIdx.z);
    const int cbase = r1 + tcol * TC_T;
    const int ncol = min(TC_T, rest - tcol * TC_T);
#pragma unroll 1
    for (int q = 0; q < TC_T / 32; ++q) {
      if (32 * q >= ncol) break;
      uint32_t vr[32], vi[32];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(32 * q);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7]),
            "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]),
            "=r"(vr[15]), "=r"(vr[16]), "=r"(vr[17]), "=r"(vr[18]), "=r"(vr[19]), "=r"(vr[20]), "=r"(vr[21]),
            "=r"(vr[22]), "=r"(vr[23]), "=r"(vr[24]), "=r"(vr[25]), "=r"(vr[26]), "=r"(vr[27]), "=r"(vr[28]),
            "=r"(vr[29]), "=r"(vr[30]), "=r"(vr[31])
          : "r"(ta));
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7]),
            "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]),
            "=r"(vi[15]), "=r"(vi[16]), "=r"(vi[17]), "=r"(vi[18]), "=r"(vi[19]), "=r"(vi[20]), "=r"(vi[21]),
            "=r"(vi[22]), "=r"(vi[23]), "=r"(vi[24]), "=r"(vi[25]), "=r"(vi[26]), "=r"(vi[27]), "=r"(vi[28]),
            "=r"(vi[29]), "=r"(vi[30]), "=r"(vi[31])
          : "r"(ta + (uint32_t)TC_T));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (gr < n) {
        float2 cur[32];
        float2* p = A + gr + (long long)n * (cbase + 32 * q);
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (32 * q + j < ncol) cur[j] = p[(long long)n * j];
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (32 * q + j < ncol) {
            float2 v = cur[j];
            v.x -= __uint_as_float(vr[j]);
            v.y -= __uint_as_float(vi[j]);
            p[(long long)n * j] = v;
          }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

// Operand images of the trailing update written by the block products'
// epilogue, for two chunks (32 complex k) of one accumulator row: vr, vi the
// row's 32 real and imaginary parts (FP32 bits), img the first chunk's image.
// An A row (L21): k-groups Re(k 0..7), Re(k 8..15), Im(k 0..7), Im(k 8..15).
__device__ __forceinline__ void tc_store_a_row(unsigned char* img, int row, const uint32_t* vr, const uint32_t* vi,
                                               int f16) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float x[4][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      x[0][j] = __uint_as_float(vr[16 * h + j]);
      x[1][j] = __uint_as_float(vr[16 * h + 8 + j]);
      x[2][j] = __uint_as_float(vi[16 * h + j]);
      x[3][j] = __uint_as_float(vi[16 * h + 8 + j]);
    }
    unsigned char* c = img + h * 2 * TC_AIMG;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      uint4 hi, lo;
      if (f16) split8<true>(x[g], hi, lo);
      else split8<false>(x[g], hi, lo);
      *reinterpret_cast<uint4*>(c + tc_row_off(row, g)) = hi;
      *reinterpret_cast<uint4*>(c + TC_AIMG + tc_row_off(row, g)) = lo;
    }
  }
}

// The two B rows of one column of U12 (mode 2's accumulator row: vr = Re,
// vi = -Im of the column's entries): [Br; -Bi] = [vr; vi] and [Bi; Br] =
// [-vi; vr], as tc_prep_kernel lays them out.
__device__ __forceinline__ void tc_store_b_rows(unsigned char* img, int row, const uint32_t* vr, const uint32_t* vi,
                                                int f16) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float re[2][8], ni[2][8], im[2][8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        re[e][j] = __uint_as_float(vr[16 * h + 8 * e + j]);
        ni[e][j] = __uint_as_float(vi[16 * h + 8 * e + j]);
        im[e][j] = -ni[e][j];
      }
    unsigned char* c = img + h * 2 * TC_BIMG;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      uint4 hi, lo;
      const float* xr = g < 2 ? re[g & 1] : ni[g & 1];
      const float* xi = g < 2 ? im[g & 1] : re[g & 1];
      if (f16) split8<true>(xr, hi, lo);
      else split8<false>(xr, hi, lo);
      *reinterpret_cast<uint4*>(c + tc_row_off(row, g)) = hi;
      *reinterpret_cast<uint4*>(c + TC_BIMG + tc_row_off(row, g)) = lo;
      if (f16) split8<true>(xi, hi, lo);
      else split8<false>(xi, hi, lo);
      *reinterpret_cast<uint4*>(c + tc_row_off(TC_T + row, g)) = hi;
      *reinterpret_cast<uint4*>(c + TC_BIMG + tc_row_off(TC_T + row, g)) = lo;
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent form of the same update: one CTA per SM walks the tiles of the
// launch (tile t, t + grid, ...) with three roles, so that one tile's
// read-modify-write of A22 runs while the next tile's MMAs do:
//   warp 0 (one thread)  streams operand chunks into TCP_STAGES shared-memory
//                        stages (bulk async copies, full/empty mbarriers);
//   warp 1 (one thread)  issues the MMAs of a tile into one of two 256-column
//                        TMEM accumulators (512 columns in all) and commits the
//                        finished accumulator to acc_full[buf];
//   warps 2-5            read the accumulator (each warp the TMEM lane quarter
//                        it may access, warp % 4), release it on acc_empty[buf]
//                        and subtract it from A22.
// Modes 1 and 2 are the panel's block products, written over their operand
// (each tile is the only reader of its operand's tile) together with the
// operand images of the trailing update, into iout:
//   mode 1: L21 = A21 V, a row tile per tile (A: A21's images, B: V's);
//   mode 2: conj(U12^T) = conj(A12^T) conj(W^T), a column tile of U12 per
//           tile: accumulator row = column of U12, so each thread writes its
//           column's B-image rows (A: the first half of A12's B images, B:
//           conj(W^T)'s image).
// Every mbarrier wait is bounded; a role that times out raises the status,
// flags the others through shared memory, and each role waits (bounded) for
// the copies or MMAs it has in flight before the CTA frees its tensor memory.
// ---------------------------------------------------------------------------
constexpr int TCP_STAGES = 4;
constexpr int TCP_THREADS = 192;
constexpr int TCP_SMEM = TCP_STAGES * TC_STAGE + 256;

__global__ void __launch_bounds__(TCP_THREADS, 1) tc_update_persistent_kernel(
    BatchT<float2> b, int k0, const unsigned char* __restrict__ abuf, const unsigned char* __restrict__ bbuf,
    long long sys_bytes_a, long long sys_bytes_b, int nt, int nsys, int* status, uint32_t idesc, int ti0, int nti,
    int tj0, int ntc, const unsigned char* __restrict__ pabuf, const unsigned char* __restrict__ pbbuf, int mode,
    unsigned char* iout, int f16) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TCP_STAGES * TC_STAGE);
  // bars: full[S], empty[S], acc_full[2], acc_empty[2]; then the TMEM address
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * TCP_STAGES + 4);
  __shared__ volatile int s_err;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[TCP_STAGES]);
  const uint32_t accf0 = smem_u32(&bars[2 * TCP_STAGES]), acce0 = smem_u32(&bars[2 * TCP_STAGES + 2]);
  const int r1 = k0 + LU_OUTER;
  const long long total = (long long)nti * ntc * nsys;
  // chunks per tile: the previous panel's images first (a merged update), then this panel's
  const int nch = pabuf ? 2 * TC_NCH : TC_NCH;
  // tile t: system z, row tile trow in [ti0, ti0 + nti), column tile tcol in
  // [tj0, tj0 + ntc); false beyond a ragged system's order
  auto tile = [&](long long t, int& z, int& trow, int& tcol) {
    z = (int)(t / ((long long)nti * ntc));
    const int rem = (int)(t % ((long long)nti * ntc));
    trow = ti0 + rem / ntc;
    tcol = tj0 + rem % ntc;
    const int rest = b.order(z) - r1;
    return rest > 0 && trow * TC_T < rest && tcol * TC_T < rest;
  };
  if (threadIdx.x == 0) {
    s_err = 0;
    for (int i = 0; i < TCP_STAGES; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * i));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8 * i));
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(accf0 + 8 * i));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(acce0 + 8 * i));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  auto fail = [&] {
    atomicCAS(status, 0, ST_TC_TIMEOUT);
    s_err = 1;
  };

  if (warp == 0 && lane == 0) {
    // producer
    const uint32_t s0 = smem_u32(smem);
    long long g = 0;   // chunks issued
    bool ok = true;
    for (long long t = blockIdx.x; t < total && ok && !s_err; t += gridDim.x) {
      int z, trow, tcol;
      if (!tile(t, z, trow, tcol)) continue;
      for (int c = 0; c < nch; ++c) {
        // the previous panel's tiles are one tile further: its trailing block starts 128 earlier
        const bool prev = pabuf && c < TC_NCH;
        const int cc = c % TC_NCH, off = prev ? 1 : 0;
        const unsigned char* ga = (prev ? pabuf : abuf) + z * sys_bytes_a +
                                  ((long long)(trow + off) * TC_NCH + cc) * 2 * TC_AIMG;
        const unsigned char* gb = (prev ? pbbuf : bbuf) + z * sys_bytes_b +
                                  ((long long)(tcol + off) * TC_NCH + cc) * 2 * TC_BIMG;
        const int q = (int)(g % TCP_STAGES);
        const long long r = g / TCP_STAGES;
        if (r > 0 && !(ok = mbar_wait(empty0 + 8 * q, (uint32_t)((r - 1) & 1)))) break;
        if (mode == 2) {   // A: rows of A12's B image (column tile tcol), B: conj(W^T) (one tile)
          const unsigned char* gt = abuf + z * sys_bytes_a + ((long long)tcol * TC_NCH + cc) * 2 * TC_BIMG;
          tc_load_chunk_split(s0 + q * TC_STAGE, gt, gt + TC_BIMG, bbuf + z * sys_bytes_b + (long long)cc * 2 * TC_BIMG,
                              full0 + 8 * q);
        } else {
          tc_load_chunk(s0 + q * TC_STAGE, ga, gb, full0 + 8 * q);
        }
        ++g;
      }
    }
    if (!ok) fail();
    // copies in flight land before the CTA can leave: the last round of each stage
    for (long long h = g - 1; h >= 0 && h >= g - TCP_STAGES; --h)
      mbar_wait(full0 + 8 * (int)(h % TCP_STAGES), (uint32_t)((h / TCP_STAGES) & 1));
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t s0 = smem_u32(smem);
    long long g = 0, i = 0;   // chunks consumed, tiles done
    bool ok = true;
    for (long long t = blockIdx.x; t < total && ok && !s_err; t += gridDim.x) {
      int z, trow, tcol;
      if (!tile(t, z, trow, tcol)) continue;
      const int buf = (int)(i & 1);
      const long long u = i >> 1;
      if (u > 0 && !(ok = mbar_wait(acce0 + 8 * buf, (uint32_t)((u - 1) & 1)))) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tm = tmem + (uint32_t)(buf * TC_TMEM_COLS);
      for (int c = 0; c < nch; ++c) {
        const int q = (int)(g % TCP_STAGES);
        if (!(ok = mbar_wait(full0 + 8 * q, (uint32_t)((g / TCP_STAGES) & 1)))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = s0 + q * TC_STAGE;
        const uint32_t ahi = st, alo = st + TC_AIMG, bhi = st + 2 * TC_AIMG, blo = bhi + TC_BIMG;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          const uint32_t o = kk * 256;
          tc_mma(tm, umma_desc(ahi + o, 128, TC_SBO), umma_desc(bhi + o, 128, TC_SBO), (c > 0 || kk > 0) ? 1u : 0u,
                 idesc);
          tc_mma(tm, umma_desc(ahi + o, 128, TC_SBO), umma_desc(blo + o, 128, TC_SBO), 1u, idesc);
          tc_mma(tm, umma_desc(alo + o, 128, TC_SBO), umma_desc(bhi + o, 128, TC_SBO), 1u, idesc);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         empty0 + 8 * q)
                     : "memory");
        ++g;
      }
      if (!ok) break;
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(accf0 + 8 * buf)
                   : "memory");
      ++i;
    }
    if (!ok) fail();
    // the MMAs issued last have completed before the tensor memory is freed
    if (g > 0) mbar_wait(empty0 + 8 * (int)((g - 1) % TCP_STAGES), (uint32_t)(((g - 1) / TCP_STAGES) & 1));
  } else if (warp >= 2) {
    // epilogue: thread = accumulator row (TMEM lane), warp w reads lanes 32 (w % 4) ..
    // (every lane waits on the barrier and the warp goes on only if all did:
    // the tcgen05.ld below must be executed by every lane of a warp)
    const int lq = warp & 3;
    const int row = lq * 32 + lane;
    long long i = 0;
    bool ok = true;
    for (long long t = blockIdx.x; t < total; t += gridDim.x) {
      if (__shfl_sync(0xffffffffu, s_err, 0)) break;
      int z, trow, tcol;
      if (!tile(t, z, trow, tcol)) continue;
      const int buf = (int)(i & 1);
      const bool got = mbar_wait(accf0 + 8 * buf, (uint32_t)((i >> 1) & 1));
      if (!(ok = __all_sync(0xffffffffu, got))) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // mode 0: A22 tile (r1 + ..., r1 + ...) -= product; mode 1: L21 tile
      // (r1 + ..., k0 + ...) = product; mode 2: U12 tile (k0 + ..., r1 + ...) = product
      const int n = b.order(z), rest = n - r1;
      // this thread's row of A22 or L21, or (mode 2) column of U12
      const int gr = r1 + (mode == 2 ? tcol : trow) * TC_T + row;
      float2* A = b.sys(z);
      const int cbase = mode == 1 ? k0 : r1 + tcol * TC_T;
      const int ncol = mode == 1 ? TC_T : min(TC_T, rest - tcol * TC_T);
#pragma unroll 1
      for (int q = 0; q < TC_T / 32; ++q) {
        uint32_t vr[32], vi[32];
        const uint32_t ta = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(buf * TC_TMEM_COLS + 32 * q);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7]),
              "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]),
              "=r"(vr[15]), "=r"(vr[16]), "=r"(vr[17]), "=r"(vr[18]), "=r"(vr[19]), "=r"(vr[20]), "=r"(vr[21]),
              "=r"(vr[22]), "=r"(vr[23]), "=r"(vr[24]), "=r"(vr[25]), "=r"(vr[26]), "=r"(vr[27]), "=r"(vr[28]),
              "=r"(vr[29]), "=r"(vr[30]), "=r"(vr[31])
            : "r"(ta));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7]),
              "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]),
              "=r"(vi[15]), "=r"(vi[16]), "=r"(vi[17]), "=r"(vi[18]), "=r"(vi[19]), "=r"(vi[20]), "=r"(vi[21]),
              "=r"(vi[22]), "=r"(vi[23]), "=r"(vi[24]), "=r"(vi[25]), "=r"(vi[26]), "=r"(vi[27]), "=r"(vi[28]),
              "=r"(vi[29]), "=r"(vi[30]), "=r"(vi[31])
            : "r"(ta + (uint32_t)TC_T));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (q == TC_T / 32 - 1) {   // every column of the accumulator is in registers: release it
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acce0 + 8 * buf) : "memory");
        }
        if (mode == 2) {   // accumulator: Re U12(k0 + k, gr) at column k, -Im U12 at 128 + k
          if (gr < n) {
            float2* p = A + (k0 + 32 * q) + (long long)n * gr;
#pragma unroll
            for (int j = 0; j < 32; ++j) p[j] = make_float2(__uint_as_float(vr[j]), -__uint_as_float(vi[j]));
          }
          tc_store_b_rows(iout + z * sys_bytes_a + ((long long)tcol * TC_NCH + 2 * q) * 2 * TC_BIMG, row, vr, vi, f16);
        } else if (gr < n && 32 * q < ncol) {
          float2* p = A + gr + (long long)n * (cbase + 32 * q);
          if (mode == 0) {
            float2 cur[32];
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (32 * q + j < ncol) cur[j] = p[(long long)n * j];
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (32 * q + j < ncol) {
                float2 v = cur[j];
                v.x -= __uint_as_float(vr[j]);
                v.y -= __uint_as_float(vi[j]);
                p[(long long)n * j] = v;
              }
          } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (32 * q + j < ncol) p[(long long)n * j] = make_float2(__uint_as_float(vr[j]), __uint_as_float(vi[j]));
          }
        }
        if (mode == 1)   // rows beyond the order are zero, as tc_prep_kernel writes them
          tc_store_a_row(iout + z * sys_bytes_a + ((long long)trow * TC_NCH + 2 * q) * 2 * TC_AIMG, row, vr, vi, f16);
      }
      ++i;
    }
    if (!ok) fail();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_TMEM_COLS));
}

// the persistent form of the update is the default; NEMOH_B200_TC_PERSISTENT=0
// selects the one-tile-per-CTA form (for comparison)
inline bool tc_persistent() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_TC_PERSISTENT");
    return !(e && e[0] == '0');
  }();
  return on;
}

// CTAs of the persistent update (one per SM): NEMOH_B200_TC_SMS caps them
// below the SM count, leaving SMs to the LU's latency-bound launches of the
// other stream groups (the update is HBM-bound, so fewer SMs may stream A22
// as fast)
inline int tc_grid_cap(int sms) {
  static const int cap = [] {
    const char* e = std::getenv("NEMOH_B200_TC_SMS");
    return e ? std::atoi(e) : 0;
  }();
  return cap > 0 ? std::min(cap, sms) : sms;
}

// operand split: BF16 terms unless NEMOH_B200_TC_SPLIT=f16 (FP16 terms).
// Measured on the barge workload (40 frequencies, N=2400): the FP16 split did
// not make the refinement converge sooner (4 passes to a relative residual of
// 3e-13 against 3 passes to 7e-13 with BF16; the factors' accuracy is bound
// by the FP32 storage and panel arithmetic, not by the split), so BF16 stays.
inline bool tc_split_f16() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_TC_SPLIT");
    return e && std::strcmp(e, "f16") == 0;
  }();
  return on;
}

// NEMOH_B200_TC=0 selects the CUDA-core FP32 update instead (for comparison)
inline bool tc_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_TC");
    return !(e && e[0] == '0');
  }();
  return on;
}

// operand images of the outer update after the panel [k0, k0+128)
inline void tc_prep(TcWork& w, BatchT<float2> b, int k0, int nsys, cudaStream_t st, long long& launches) {
  const int n = b.n, rest = n - k0 - LU_OUTER;
  if (rest <= 0) return;
  const int t = (n + TC_T - 1) / TC_T;
  const long long sa = (long long)t * TC_NCH * 2 * TC_AIMG, sb = (long long)t * TC_NCH * 2 * TC_BIMG;
  const int nt = (rest + TC_T - 1) / TC_T;
  const int per = (nt * TC_T * TC_NCH + 127) / 128;
  if (tc_split_f16()) tc_prep_kernel<true><<<dim3(2 * per, 1, nsys), 128, 0, st>>>(b, k0, w.a, w.b, sa, sb, per);
  else tc_prep_kernel<false><<<dim3(2 * per, 1, nsys), 128, 0, st>>>(b, k0, w.a, w.b, sa, sb, per);
  ++launches;
}

// A rectangle of tiles of the trailing matrix: row tiles [ti0, ti0 + nti),
// column tiles [tj0, tj0 + ntc) (a count < 0: to the last tile)
struct TcTiles {
  int ti0 = 0, nti = -1, tj0 = 0, ntc = -1;
};

// The update of a rectangle of tiles of the trailing matrix from the images
// tc_prep wrote; persistent: one CTA per SM walking the tiles (the default
// form), else one tile per CTA. prev (persistent form only): the images of
// the previous panel, whose update of these tiles was deferred and is merged
// here (K = 256 in one accumulation: one read-modify-write of the tiles for
// two panels).
inline void tc_apply(TcWork& w, BatchT<float2> b, int k0, int nsys, cudaStream_t st, long long& launches,
                     int* status, TcTiles tl, bool persistent, const TcWork* prev = nullptr) {
  const int n = b.n, rest = n - k0 - LU_OUTER;
  if (rest <= 0) return;
  const int t = (n + TC_T - 1) / TC_T;
  const long long sa = (long long)t * TC_NCH * 2 * TC_AIMG, sb = (long long)t * TC_NCH * 2 * TC_BIMG;
  const int nt = (rest + TC_T - 1) / TC_T;
  const int nti = std::min(tl.nti < 0 ? nt - tl.ti0 : tl.nti, nt - tl.ti0);
  const int ntc = std::min(tl.ntc < 0 ? nt - tl.tj0 : tl.ntc, nt - tl.tj0);
  if (nti <= 0 || ntc <= 0) return;
  const uint32_t idesc = tc_idesc(tc_split_f16());
  if (persistent || prev) {
    static std::atomic<unsigned long long> attr2{0};
    static int sms = 0;
    once_per_device(attr2, [] {
      cudaFuncSetAttribute(tc_update_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TCP_SMEM);
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    });
    const long long tiles = (long long)nti * ntc * nsys;
    const int grid = (int)std::min<long long>(tiles, tc_grid_cap(sms > 0 ? sms : 148));
    tc_update_persistent_kernel<<<grid, TCP_THREADS, TCP_SMEM, st>>>(
        b, k0, w.a, w.b, sa, sb, nt, nsys, status, idesc, tl.ti0, nti, tl.tj0, ntc, prev ? prev->a : nullptr,
        prev ? prev->b : nullptr, 0, nullptr, 0);
  } else {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
      cudaFuncSetAttribute(tc_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    });
    tc_update_kernel<<<dim3(ntc, nti, nsys), 128, TC_SMEM, st>>>(b, k0, w.a, w.b, sa, sb, status, idesc, tl.ti0,
                                                                 tl.tj0);
  }
  ++launches;
}

// The panel's block products on the tensor cores (persistent form), from
// the images tc_prep wrote of A21 and A12 before them: L21 = A21 V (every row
// tile, one column tile) and U12 = W A12 (one row tile, every column tile),
// each written over its operand; W and V from the panel's inverses
// (panel_inv_kernel). Both write the trailing update's operand images of the
// products over the operands' images (the update needs no tc_prep after).
inline void tc_products(TcWork& w, BatchT<float2> b, int k0, int nsys, cudaStream_t st, long long& launches,
                        int* status) {
  const int n = b.n, rest = n - k0 - LU_OUTER;
  if (rest <= 0) return;
  const int t = (n + TC_T - 1) / TC_T;
  const long long sa = (long long)t * TC_NCH * 2 * TC_AIMG, sb = (long long)t * TC_NCH * 2 * TC_BIMG;
  const int nt = (rest + TC_T - 1) / TC_T;
  constexpr int PER = TC_T * TC_NCH / 128;
  if (tc_split_f16()) tc_prep_wv_kernel<true><<<dim3(2 * PER, 1, nsys), 128, 0, st>>>(b, k0, w.wv);
  else tc_prep_wv_kernel<false><<<dim3(2 * PER, 1, nsys), 128, 0, st>>>(b, k0, w.wv);
  ++launches;
  const uint32_t idesc = tc_idesc(tc_split_f16());
  static std::atomic<unsigned long long> attr{0};
  static int sms = 0;
  once_per_device(attr, [] {
    cudaFuncSetAttribute(tc_update_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TCP_SMEM);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  });
  const int cap = tc_grid_cap(sms > 0 ? sms : 148);
  const int f16 = tc_split_f16() ? 1 : 0;
  // L21 = A21 V: A images of A21 (row tiles), the B image of V (tile 0)
  tc_update_persistent_kernel<<<(int)std::min<long long>((long long)nt * nsys, cap), TCP_THREADS, TCP_SMEM, st>>>(
      b, k0, w.a, w.wv + TC_W_BYTES, sa, TC_WV_BYTES, nt, nsys, status, idesc, 0, nt, 0, 1, nullptr, nullptr, 1, w.a,
      f16);
  // conj(U12^T) = conj(A12^T) conj(W^T): A from the B images of A12 (column
  // tiles), B the image of conj(W^T) (tile 0)
  tc_update_persistent_kernel<<<(int)std::min<long long>((long long)nt * nsys, cap), TCP_THREADS, TCP_SMEM, st>>>(
      b, k0, w.b, w.wv, sb, TC_WV_BYTES, nt, nsys, status, idesc, 0, 1, 0, nt, nullptr, nullptr, 2, w.b, f16);
  launches += 2;
}

}  // namespace nb200
