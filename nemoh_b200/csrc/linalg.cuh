// Dense complex FP64 linear algebra for the BEM systems (sm_100a).
//
// The reference inverts each influence matrix with GAUSSZ (Gauss elimination
// on [A|I] without effective row pivoting, Solver/Core/M_SOLVER.f90:31-104).
// Here each matrix is factored once as A = L U (L unit lower, U upper) with a
// blocked right-looking algorithm and the same no-pivot semantics, including
// the "pivot below 1e-20" stop (M_SOLVER.f90:49-52, 61-64) as a status code.
// Without pivoting a step of width 32 reduces to the small diagonal block and
// two block products with its inverses (blockIdx.z = system):
//   lu_diag_kernel    factor A11 once per system, invert L11 and U11
//   lu_panel_kernel   L21 <- A21 U11^-1, U12 <- L11^-1 A12, store factored A11
//   zgemm_update      A22 <- A22 - L21 U12 over any rectangle of A22
// The FP64 path updates the whole trailing matrix after every step; the mixed
// path (mixed.cuh) defers the update outside a 128-column panel to one
// tensor-core product per panel.
#pragma once
#include <cooperative_groups.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "common.cuh"

namespace nb200 {

constexpr int LU_NB = 32;     // panel width
constexpr int LU_RB = 128;    // rows per L21 CTA
constexpr int LU_CB = 64;     // columns per U12 CTA

// A batch of systems. Uniform: every system has order n and starts `stride`
// elements after the previous one. Ragged (systems of different bodies in one
// launch sequence): `off` and `ord` (device arrays) give each system's offset
// and order, n is the largest order, and the systems are sorted by decreasing
// order so that the systems still active at an elimination step are a prefix
// of the batch; every kernel takes its own system's order and leaves the parts
// of the launch grid beyond it. Per-system scratch (diag, pinv, inverted
// diagonal blocks, right-hand sides) keeps uniform strides sized by n.
template <class C2>
struct BatchT {
  C2* base;               // system s at base + s * stride (uniform) or base + off[s] (ragged)
  long long stride;       // elements between systems (uniform)
  int n;                  // order (uniform), largest order (ragged)
  C2* diag;               // DIAG_SCRATCH elements per system: factored A11, inv(L11), inv(U11)
  C2* pinv = nullptr;     // optional, PINV_SCRATCH per system: inv(L) of the LU_OUTER / LU_NB
                          // diagonal blocks of the current outer panel (two-level LU only)
  const long long* off = nullptr;   // ragged: element offset of each system
  const int* ord = nullptr;         // ragged: order (and leading dimension) of each system
  __device__ __forceinline__ int order(int s) const { return ord ? ord[s] : n; }
  __device__ __forceinline__ C2* sys(int s) const { return base + (off ? off[s] : (long long)s * stride); }
};
// The ragged description of a batch: device arrays for the kernels, and the
// orders again on the host (decreasing) for the launch loop.
struct Ragged {
  const long long* off = nullptr;
  const int* ord = nullptr;
  const int* host_ord = nullptr;
  const long long* host_off = nullptr;   // host copy of off
};
template <class C2>
inline BatchT<C2> make_batch(C2* base, int n, C2* diag, C2* pinv, const Ragged& rg) {
  BatchT<C2> b{base, (long long)n * n, n, diag, pinv};
  b.off = rg.off;
  b.ord = rg.ord;
  return b;
}
constexpr int DIAG_SCRATCH = 3 * LU_NB * LU_NB;
constexpr int LU_OUTER = 128;
// per system, for the current outer panel: inv(L) of its LU_OUTER / LU_NB
// diagonal blocks (P), inv(U) of the same blocks (Q), then inv(L11) (W) and
// inv(U11) (V) of the whole panel (LU_OUTER x LU_OUTER, column-major)
constexpr int PINV_DIAG = (LU_OUTER / LU_NB) * LU_NB * LU_NB;
constexpr int PINV_Q_OFF = PINV_DIAG;
constexpr int PINV_W_OFF = 2 * PINV_DIAG;
constexpr int PINV_V_OFF = PINV_W_OFF + LU_OUTER * LU_OUTER;
constexpr int PINV_SCRATCH = PINV_V_OFF + LU_OUTER * LU_OUTER;
using Batch = BatchT<double2>;

template <class C2> __device__ __forceinline__ C2 mkc(double x, double y);
template <> __device__ __forceinline__ double2 mkc<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 mkc<float2>(double x, double y) { return make_float2((float)x, (float)y); }

template <class C2>
__device__ __forceinline__ C2 cfms(C2 c, C2 a, C2 b) {  // c - a*b
  C2 r;
  r.x = c.x - (a.x * b.x - a.y * b.y);
  r.y = c.y - (a.x * b.y + a.y * b.x);
  return r;
}
__device__ __forceinline__ double2 cdv(double2 a, double2 b) {
  cplx r = mk(a.x, a.y) / mk(b.x, b.y);
  return make_double2(r.re, r.im);
}
__device__ __forceinline__ float2 cdv(float2 a, float2 b) {
  if (fabsf(b.x) >= fabsf(b.y)) {
    float r = b.y / b.x, d = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  float r = b.x / b.y, d = b.y + b.x * r;
  return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double cabs2(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double cabs2(float2 a) { return hypotf(a.x, a.y); }

// Factor the diagonal block A11 of step k once per system (grid.z = system)
// and invert its triangles. Scratch per system: [LU(A11) | inv(L11) | inv(U11)],
// column-major nb x nb each (ld = nb). One thread per element of the 32 x 32
// block, every step of the three eliminations separated by a barrier:
//  * unpivoted Doolittle (GAUSSZ's elimination on this block): at step j the
//    column below the pivot is divided by it, then the trailing block takes
//    the rank-1 update;
//  * inv(L): X = I, step j (ascending) subtracts L(i, j) X(j, :) from the rows
//    below, the order of the column-by-column forward substitution;
//  * inv(U): X = I, step j (descending) divides row j by U(j, j) and
//    subtracts U(i, j) X(j, :) from the rows above.
// With b.pinv (two-level LU) inv(L) also goes to the slot of this block in the
// current outer panel. (Measured against two 128-thread forms, warp-owned
// columns with the inverses either by warp-owned columns or one column per
// lane in registers: 28.6 us per launch here against 78.5 and 65 us; the
// register form's long unrolled instruction stream stalls on instruction
// fetch.)
constexpr int LU_DIAG_THREADS = LU_NB * LU_NB;
template <class C2>
__global__ void __launch_bounds__(LU_DIAG_THREADS) lu_diag_kernel(BatchT<C2> b, int k, int* status) {
  __shared__ C2 sb[LU_NB * LU_NB];   // the block, column-major, ld = nb
  __shared__ C2 xl[LU_NB * LU_NB];   // inv(L11), ld = LU_NB
  __shared__ C2 xu[LU_NB * LU_NB];   // inv(U11), ld = LU_NB
  const int n = b.order(blockIdx.z);
  if (k >= n) return;
  const int nb = min(LU_NB, n - k);
  const int i = threadIdx.x & (LU_NB - 1), c = threadIdx.x / LU_NB;
  const bool in = i < nb && c < nb;
  const C2* A = b.sys(blockIdx.z);
  if (in) sb[i + nb * c] = A[(k + i) + (long long)n * (k + c)];
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (threadIdx.x == 0 && !(cabs2(sb[j + nb * j]) > 1.E-20)) atomicCAS(status, 0, ST_PIVOT);
    if (in && c == j && i > j) sb[i + nb * j] = cdv(sb[i + nb * j], sb[j + nb * j]);
    __syncthreads();
    if (in && i > j && c > j) sb[i + nb * c] = cfms(sb[i + nb * c], sb[i + nb * j], sb[j + nb * c]);
    __syncthreads();
  }
  const C2 one = mkc<C2>(1., 0.), zero = mkc<C2>(0., 0.);
  if (in) {
    xl[i + LU_NB * c] = i == c ? one : zero;
    xu[i + LU_NB * c] = i == c ? one : zero;
  }
  __syncthreads();
  for (int step = 0; step < nb; ++step) {
    const int jl = step, ju = nb - 1 - step;
    if (in && i == ju && c >= ju) xu[ju + LU_NB * c] = cdv(xu[ju + LU_NB * c], sb[ju + nb * ju]);
    __syncthreads();
    if (in && i > jl && c <= jl) xl[i + LU_NB * c] = cfms(xl[i + LU_NB * c], sb[i + nb * jl], xl[jl + LU_NB * c]);
    if (in && i < ju && c >= ju) xu[i + LU_NB * c] = cfms(xu[i + LU_NB * c], sb[i + nb * ju], xu[ju + LU_NB * c]);
    __syncthreads();
  }
  C2* D = b.diag + (long long)blockIdx.z * DIAG_SCRATCH;
  C2* P = b.pinv ? b.pinv + (long long)blockIdx.z * PINV_SCRATCH + ((k % LU_OUTER) / LU_NB) * LU_NB * LU_NB : nullptr;
  if (in) {
    const int q = i + nb * c;
    D[q] = sb[q];
    D[LU_NB * LU_NB + q] = xl[i + LU_NB * c];
    D[2 * LU_NB * LU_NB + q] = xu[i + LU_NB * c];
    if (P) P[q] = xl[i + LU_NB * c];
  }
}

// acc += a b as four fused multiply-adds into the accumulator (written out:
// `acc.x += a.x*b.x - a.y*b.y` compiles to a multiply, an FMA and an add per
// component, 50% more floating-point instructions in the update loops)
__device__ __forceinline__ double fmx(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmx(float a, float b, float c) { return fmaf(a, b, c); }
// two consecutive complex values of shared memory (the first at an even
// index: one 16-byte load in single precision)
__device__ __forceinline__ void ld_pair(const float2* p, float2& a, float2& b) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void ld_pair(const double2* p, double2& a, double2& b) {
  a = p[0];
  b = p[1];
}

template <class C2>
__device__ __forceinline__ void cmac(C2& acc, C2 a, C2 b) {
  acc.x = fmx(a.x, b.x, acc.x);
  acc.x = fmx(-a.y, b.y, acc.x);
  acc.y = fmx(a.x, b.y, acc.y);
  acc.y = fmx(a.y, b.x, acc.y);
}

// L21 <- A21 inv(U11) (CTAs [0, nrb), one thread per row) and
// U12 <- inv(L11) A12 for the columns [k + nb, ucol_end) (CTAs [nrb, nrb+ncb),
// one lane per row of a column), with the
// inverses from lu_diag_kernel; CTA 0 also stores the factored A11 into A
// (no kernel of the step reads A11 from A). Launch with at least one CTA.
template <class C2>
__global__ void __launch_bounds__(LU_RB) lu_panel_kernel(BatchT<C2> b, int k, int ucol_end) {
  __shared__ C2 inv[LU_NB * LU_NB];
  __shared__ C2 work[LU_NB * LU_CB];
  const int n = b.order(blockIdx.z);
  if (k >= n) return;
  ucol_end = min(ucol_end, n);
  const int nb = min(LU_NB, n - k);
  C2* A = b.sys(blockIdx.z);
  const C2* D = b.diag + (long long)blockIdx.z * DIAG_SCRATCH;
  const int rest = n - k - nb;
  const int nrb = (rest + LU_RB - 1) / LU_RB;
  if (blockIdx.x == 0)
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) A[(k + q % nb) + (long long)n * (k + q / nb)] = D[q];
  if (blockIdx.x < nrb) {
    for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) inv[q] = D[2 * LU_NB * LU_NB + q];
    __syncthreads();
    const int r = k + nb + blockIdx.x * LU_RB + threadIdx.x;
    if (r >= n) return;
    C2 x[LU_NB];
#pragma unroll
    for (int c = 0; c < LU_NB; ++c)
      x[c] = (c < nb) ? A[r + (long long)n * (k + c)] : mkc<C2>(0., 0.);
    // out(c) = sum_{j <= c} x(j) invU(j, c)
#pragma unroll
    for (int c = 0; c < LU_NB; ++c) {
      if (c < nb) {
        C2 acc = mkc<C2>(0., 0.);
#pragma unroll
        for (int j = 0; j <= c; ++j) cmac(acc, x[j], inv[j + nb * c]);
        A[r + (long long)n * (k + c)] = acc;
      }
    }
    return;
  }
  for (int q = threadIdx.x; q < nb * nb; q += blockDim.x) inv[q] = D[LU_NB * LU_NB + q];
  const int c0 = k + nb + (blockIdx.x - nrb) * LU_CB;
  const int ncol = min(LU_CB, ucol_end - c0);
  for (int q = threadIdx.x; q < nb * ncol; q += blockDim.x) {
    const int i = q % nb, c = q / nb;
    work[i + nb * c] = A[(k + i) + (long long)n * (c0 + c)];
  }
  __syncthreads();
  // y(i, c) = a(i, c) + sum_{j < i} invL(i, j) a(j, c): lane = row i, the
  // CTA's four warps take every fourth column; results go straight to A
  const int i = threadIdx.x & 31;
  if (i >= nb) return;
  for (int c = threadIdx.x >> 5; c < ncol; c += LU_RB / 32) {
    const C2* a = work + nb * c;
    C2 acc = a[i];
    for (int j = 0; j < i; ++j) cmac(acc, inv[i + nb * j], a[j]);
    A[(k + i) + (long long)n * (c0 + c)] = acc;
  }
}

// A[r0:r1, c0:c1] -= A[r0:r1, k:k+kb] A[k:k+kb, c0:c1]: 64 x 64 output tile
// per CTA (grid.x over columns, grid.y over rows), 128 threads; thread
// (tr, tc) = (t % 16, t / 16) owns rows tr + 16 i (i < 4) and columns
// 8 tc + j (j < 8), so 16 consecutive lanes own 16 consecutive rows of a
// column (coalesced read-modify-write of the result) while each k step reads
// 4 A values (contiguous across lanes) and 8 B values (broadcast) from shared
// memory for 32 complex FMAs. The inner dimension streams through two
// shared-memory stages of 16 with asynchronous copies (cp.async, zero-filled
// outside the operands), so the next chunk loads while the current one is
// multiplied; B rows are padded to 65 elements against bank conflicts.
constexpr int GM_T = 64;
constexpr int GM_BS = GM_T + 1;
constexpr int GM_KC = 16;
struct Rect {
  int r0, r1, c0, c1;
};
template <class C2>
constexpr int zgemm_smem() {
  return 2 * (GM_KC * GM_T + GM_KC * GM_BS) * (int)sizeof(C2);
}

// asynchronous global -> shared copy of one complex element; src_bytes = 0
// zero-fills the destination without reading
template <class C2>
__device__ __forceinline__ void cp_async_elem(C2* dst, const C2* src, bool valid) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  const int nbytes = valid ? (int)sizeof(C2) : 0;
  if (sizeof(C2) == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(nbytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(nbytes) : "memory");
}

template <class C2>
__global__ void __launch_bounds__(128) zgemm_update_kernel(BatchT<C2> b, int k, int kb, Rect rc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2* stage0 = reinterpret_cast<C2*>(smem_raw);
  constexpr int STAGE = GM_KC * GM_T + GM_KC * GM_BS;   // As [16][64] then Bs [16][65]
  const int n = b.order(blockIdx.z);
  rc.r1 = min(rc.r1, n);
  rc.c1 = min(rc.c1, n);
  kb = min(kb, n - k);
  const int r0 = rc.r0 + blockIdx.y * GM_T;
  const int c0 = rc.c0 + blockIdx.x * GM_T;
  if (r0 >= rc.r1 || c0 >= rc.c1 || kb <= 0) return;
  C2* A = b.sys(blockIdx.z);
  const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
  auto load = [&](int s, int k0) {
    C2* As = stage0 + s * STAGE;
    C2* Bs = As + GM_KC * GM_T;
    const int kc = min(GM_KC, kb - k0);
    for (int q = threadIdx.x; q < GM_KC * GM_T; q += 128) {
      const int m = q % GM_T, kk = q / GM_T;
      const int r = r0 + m;
      const bool v = r < rc.r1 && kk < kc;
      cp_async_elem(As + kk * GM_T + m, v ? A + r + (long long)n * (k + k0 + kk) : A, v);
    }
    for (int q = threadIdx.x; q < GM_KC * GM_T; q += 128) {
      const int kk = q % GM_KC, nn = q / GM_KC;
      const int c = c0 + nn;
      const bool v = c < rc.c1 && kk < kc;
      cp_async_elem(Bs + kk * GM_BS + nn, v ? A + (k + k0 + kk) + (long long)n * c : A, v);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  C2 acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = mkc<C2>(0., 0.);
  load(0, 0);
  int s = 0;
  for (int k0 = 0; k0 < kb; k0 += GM_KC, s ^= 1) {
    const bool more = k0 + GM_KC < kb;
    if (more) {
      load(s ^ 1, k0 + GM_KC);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const C2* As = stage0 + s * STAGE;
    const C2* Bs = As + GM_KC * GM_T;
#pragma unroll 2
    for (int kk = 0; kk < GM_KC; ++kk) {
      C2 a[4], bb[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk * GM_T + tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) bb[j] = Bs[kk * GM_BS + 8 * tc + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) cmac(acc[i][j], a[i], bb[j]);
    }
    __syncthreads();   // stage s is refilled two chunks later
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = c0 + 8 * tc + j;
    if (c >= rc.c1) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = r0 + tr + 16 * i;
      if (r >= rc.r1) continue;
      C2* p = A + r + (long long)n * c;
      C2 v = *p;
      v.x -= acc[i][j].x;
      v.y -= acc[i][j].y;
      *p = v;
    }
  }
}

template <class C2>
inline void zgemm_update(BatchT<C2> b, int k, int kb, Rect rc, int nsys, cudaStream_t st) {
  if (rc.r1 <= rc.r0 || rc.c1 <= rc.c0) return;
  const dim3 grid((rc.c1 - rc.c0 + GM_T - 1) / GM_T, (rc.r1 - rc.r0 + GM_T - 1) / GM_T, nsys);
  zgemm_update_kernel<C2><<<grid, 128, zgemm_smem<C2>(), st>>>(b, k, kb, rc);
}

// Two-level blocked LU of nsys systems (grid.z = system). Panels of LU_OUTER
// columns are factored with LU_NB-column steps whose updates stay inside the
// panel (all rows below) and the panel's row strip (all columns right of it);
// the rest of the trailing matrix is updated once per panel by `outer(k0,
// kend)`, A[kend:, kend:] -= A[kend:, k0:kend] A[k0:kend, kend:], which cuts
// the trailing matrix's read-modify-write traffic by LU_OUTER / LU_NB.
// Row strip of an outer panel: U[k0:kend, kend:n] = inv(L11) A[k0:kend, kend:n]
// with L11 the unit-lower part of the factored panel's diagonal block, by
// blocks of LU_NB rows: X_j <- inv(L_jj) X_j (inverses from lu_diag, in
// b.pinv), then X_i -= L_ij X_j for the blocks below. CTA = one system and
// ST_C columns of the strip, held in shared memory (column-major, ld
// LU_OUTER); thread = (row i of a block, every fourth column). Replaces the
// per-step row-strip updates of the right-looking panel factorization, so the
// strip is read and written once per outer panel.
constexpr int ST_C = 32;
template <class C2>
constexpr int strip_smem() {
  return (LU_OUTER * ST_C + LU_NB * LU_NB + LU_NB * ST_C) * (int)sizeof(C2);
}
template <class C2>
__global__ void __launch_bounds__(128) strip_kernel(BatchT<C2> b, int k0) {
  extern __shared__ __align__(16) unsigned char strip_sm[];
  C2* X = reinterpret_cast<C2*>(strip_sm);   // [ST_C][LU_OUTER]
  C2* T = X + LU_OUTER * ST_C;              // [LU_NB][LU_NB] inv(L_jj) or L_ij, column-major
  C2* Y = T + LU_NB * LU_NB;                // [ST_C][LU_NB]
  const int n = b.order(blockIdx.z), kend = k0 + LU_OUTER;
  const int c0 = kend + blockIdx.x * ST_C, ncol = min(ST_C, n - c0);
  if (ncol <= 0) return;
  C2* A = b.sys(blockIdx.z);
  const C2* P = b.pinv + (long long)blockIdx.z * PINV_SCRATCH;
  for (int q = threadIdx.x; q < LU_OUTER * ST_C; q += blockDim.x) {
    const int r = q % LU_OUTER, c = q / LU_OUTER;
    X[q] = c < ncol ? A[(k0 + r) + (long long)n * (c0 + c)] : mkc<C2>(0., 0.);
  }
  const int i = threadIdx.x & (LU_NB - 1), g = threadIdx.x / LU_NB;
  constexpr int NBLK = LU_OUTER / LU_NB, GROUPS = 128 / LU_NB;
  for (int jb = 0; jb < NBLK; ++jb) {
    __syncthreads();
    for (int q = threadIdx.x; q < LU_NB * LU_NB; q += blockDim.x) T[q] = P[jb * LU_NB * LU_NB + q];
    __syncthreads();
    // Y = inv(L_jj) X_j (unit diagonal); each inverse entry is read once and
    // applied to the thread's ST_C / GROUPS columns
    {
      constexpr int CPT = ST_C / GROUPS;
      C2 acc[CPT];
#pragma unroll
      for (int m = 0; m < CPT; ++m) acc[m] = X[(g + GROUPS * m) * LU_OUTER + jb * LU_NB + i];
      for (int j = 0; j < LU_NB; ++j) {
        if (j >= i) break;
        const C2 t = T[i + LU_NB * j];
#pragma unroll
        for (int m = 0; m < CPT; ++m) cmac(acc[m], t, X[(g + GROUPS * m) * LU_OUTER + jb * LU_NB + j]);
      }
#pragma unroll
      for (int m = 0; m < CPT; ++m) Y[(g + GROUPS * m) * LU_NB + i] = acc[m];
    }
    __syncthreads();
    for (int c = g; c < ST_C; c += GROUPS) {
      const C2 v = Y[c * LU_NB + i];
      X[c * LU_OUTER + jb * LU_NB + i] = v;
      if (c < ncol) A[(k0 + jb * LU_NB + i) + (long long)n * (c0 + c)] = v;
    }
    // X_i -= L_ij X_j for the blocks below
    for (int ib = jb + 1; ib < NBLK; ++ib) {
      __syncthreads();
      for (int q = threadIdx.x; q < LU_NB * LU_NB; q += blockDim.x) {
        const int r = q % LU_NB, cc = q / LU_NB;
        T[q] = A[(k0 + ib * LU_NB + r) + (long long)n * (k0 + jb * LU_NB + cc)];
      }
      __syncthreads();
      constexpr int CPT = ST_C / GROUPS;
      C2 acc[CPT];
#pragma unroll
      for (int m = 0; m < CPT; ++m) acc[m] = mkc<C2>(0., 0.);
      for (int j = 0; j < LU_NB; ++j) {
        const C2 t = T[i + LU_NB * j];
#pragma unroll
        for (int m = 0; m < CPT; ++m) cmac(acc[m], t, X[(g + GROUPS * m) * LU_OUTER + jb * LU_NB + j]);
      }
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        C2& y = X[(g + GROUPS * m) * LU_OUTER + ib * LU_NB + i];
        y.x -= acc[m].x;
        y.y -= acc[m].y;
      }
    }
  }
}

// The row strip as a product, U[k0:kend, kend:n] = W A[k0:kend, kend:n] with
// W = inv(L11) formed once per panel and system (strip_winv_kernel): the
// strip's blocks no longer wait on one another, so every block of W a CTA
// needs can be in flight at once.
//
// strip_winv_kernel: one CTA per system, thread = element (r, c) of a 32 x 32
// block. Column block j of W: W_jj = inv(L_jj) (from lu_diag), then for the
// blocks below W_ij = -inv(L_ii) sum_{k=j}^{i-1} L_ik W_kj.
constexpr int SW_BLK = LU_OUTER / LU_NB;
template <class C2>
constexpr int strip_winv_smem() {   // a column block of W, the sum S, the L11 blocks below the diagonal, inv(L_ii)
  return (SW_BLK * LU_NB * LU_NB + LU_NB * LU_NB + (SW_BLK * (SW_BLK - 1) / 2) * LU_NB * LU_NB +
          SW_BLK * LU_NB * LU_NB) * (int)sizeof(C2);
}
template <class C2>
__device__ __forceinline__ void strip_winv_body(const BatchT<C2>& b, int k0) {
  extern __shared__ __align__(16) unsigned char sw_sm[];
  constexpr int BB = LU_NB * LU_NB;
  C2* Wc = reinterpret_cast<C2*>(sw_sm);   // [SW_BLK][BB] column block j of W, column-major blocks
  C2* S = Wc + SW_BLK * BB;                // [BB]
  C2* Ls = S + BB;                         // L_ik (i > k) at ((i (i - 1)) / 2 + k) * BB
  C2* Ps = Ls + (SW_BLK * (SW_BLK - 1) / 2) * BB;   // inv(L_ii) at i * BB
  const int n = b.order(blockIdx.z);
  if (k0 + LU_OUTER >= n) return;
  const C2* A = b.sys(blockIdx.z);
  const C2* P = b.pinv + (long long)blockIdx.z * PINV_SCRATCH;
  C2* W = b.pinv + (long long)blockIdx.z * PINV_SCRATCH + PINV_W_OFF;
  const int r = threadIdx.x % LU_NB, c = threadIdx.x / LU_NB, e = r + LU_NB * c;
  // every block this system needs, loaded once (coalesced along the rows)
  for (int i = 1; i < SW_BLK; ++i)
    for (int k = 0; k < i; ++k)
      Ls[((i * (i - 1)) / 2 + k) * BB + e] = A[(k0 + i * LU_NB + r) + (long long)n * (k0 + k * LU_NB + c)];
  for (int i = 0; i < SW_BLK; ++i) Ps[i * BB + e] = P[i * BB + e];
  for (int j = 0; j < SW_BLK; ++j) {
    __syncthreads();   // the staged blocks (first pass) and the previous column block's stores are done
    Wc[j * BB + e] = Ps[j * BB + e];
    for (int i = j + 1; i < SW_BLK; ++i) {
      __syncthreads();   // W_kj for k < i are in shared memory
      C2 acc = mkc<C2>(0., 0.);
      for (int k = j; k < i; ++k) {
        const C2* L = Ls + ((i * (i - 1)) / 2 + k) * BB + r;
        const C2* Wk = Wc + k * BB + LU_NB * c;
#pragma unroll 8
        for (int m = 0; m < LU_NB; ++m) cmac(acc, L[LU_NB * m], Wk[m]);
      }
      S[e] = acc;
      __syncthreads();
      const C2* Pi = Ps + i * BB + r;
      C2 w = mkc<C2>(0., 0.);
#pragma unroll 8
      for (int m = 0; m < LU_NB; ++m) cmac(w, Pi[LU_NB * m], S[m + LU_NB * c]);
      Wc[i * BB + e] = mkc<C2>(-w.x, -w.y);
    }
    __syncthreads();
    for (int i = j; i < SW_BLK; ++i) W[(i * LU_NB + r) + LU_OUTER * (j * LU_NB + c)] = Wc[i * BB + e];
  }
}

// strip_gemm_kernel: CTA = one system and ST_C columns of the strip (held in
// shared memory, column-major, ld LU_OUTER); thread = (row i of a block, every
// fourth column). The ten nonzero 32 x 32 blocks of W stream through two
// shared buffers (cp.async, the next one in flight while the current one is
// applied); output block ib = sum_{jb <= ib} W_ib,jb X_jb goes straight to A.
template <class C2>
constexpr int strip_gemm_smem() {
  return (LU_OUTER * ST_C + 2 * LU_NB * LU_NB) * (int)sizeof(C2);
}
template <class C2>
__device__ __forceinline__ void strip_gemm_body(const BatchT<C2>& b, int k0, int bx) {
  extern __shared__ __align__(16) unsigned char sg_sm[];
  C2* X = reinterpret_cast<C2*>(sg_sm);   // [ST_C][LU_OUTER] the strip before the solve
  C2* Wb = X + LU_OUTER * ST_C;           // [2][LU_NB][LU_NB] blocks of W, column-major
  const int n = b.order(blockIdx.z), kend = k0 + LU_OUTER;
  const int c0 = kend + bx * ST_C, ncol = min(ST_C, n - c0);
  if (ncol <= 0) return;
  C2* A = b.sys(blockIdx.z);
  const C2* W = b.pinv + (long long)blockIdx.z * PINV_SCRATCH + PINV_W_OFF;
  // block step s -> (ib, jb): (0,0), (1,0), (1,1), (2,0), ...
  auto blk = [](int s, int& ib, int& jb) {
    ib = 0;
    while ((ib + 1) * (ib + 2) / 2 <= s) ++ib;
    jb = s - ib * (ib + 1) / 2;
  };
  auto fetch = [&](int s) {
    int ib, jb;
    blk(s, ib, jb);
    C2* dst = Wb + (s & 1) * LU_NB * LU_NB;
    for (int q = threadIdx.x; q < LU_NB * LU_NB; q += blockDim.x) {
      const int rr = q % LU_NB, cc = q / LU_NB;
      cp_async_elem(dst + q, W + (ib * LU_NB + rr) + LU_OUTER * (jb * LU_NB + cc), true);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  fetch(0);
  for (int q = threadIdx.x; q < LU_OUTER * ST_C; q += blockDim.x) {
    const int rr = q % LU_OUTER, cc = q / LU_OUTER;
    X[q] = cc < ncol ? A[(k0 + rr) + (long long)n * (c0 + cc)] : mkc<C2>(0., 0.);
  }
  const int i = threadIdx.x & (LU_NB - 1), g = threadIdx.x / LU_NB;
  constexpr int GROUPS = 128 / LU_NB, CPT = ST_C / GROUPS, NSTEP = SW_BLK * (SW_BLK + 1) / 2;
  C2 acc[CPT];
  for (int s = 0; s < NSTEP; ++s) {
    int ib, jb;
    blk(s, ib, jb);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();   // block s has landed; every thread is done with block s - 1
    if (s + 1 < NSTEP) fetch(s + 1);
    if (jb == 0) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) acc[m] = mkc<C2>(0., 0.);
    }
    const C2* T = Wb + (s & 1) * LU_NB * LU_NB;
    for (int j = 0; j < LU_NB; j += 2) {   // two k at a time: one 16-byte load gives both strip entries
      const C2 t0 = T[i + LU_NB * j], t1 = T[i + LU_NB * (j + 1)];
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        C2 x0, x1;
        ld_pair(X + (g + GROUPS * m) * LU_OUTER + jb * LU_NB + j, x0, x1);
        cmac(acc[m], t0, x0);
        cmac(acc[m], t1, x1);
      }
    }
    if (jb == ib) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int c = g + GROUPS * m;
        if (c < ncol) A[(k0 + ib * LU_NB + i) + (long long)n * (c0 + c)] = acc[m];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Panel of the FP32 LU as one block (mixed path): instead of LU_OUTER / LU_NB
// steps of (diagonal block, panel, in-panel update) launches,
//   panel_block_kernel    factors the panel's LU_OUTER x LU_OUTER diagonal
//                         block A11 in shared memory (GAUSSZ's unpivoted
//                         elimination) and inverts the triangles of its 32 x 32
//                         diagonal blocks (P = inv(L_ii), Q = inv(U_ii));
//   panel_inv_kernel      W = inv(L11) and V = inv(U11), one CTA each per system;
//   panel_products_kernel L21 = A21 V for every row below the panel and
//                         U12 = W A12 for the row strip, in one launch;
// then the outer update as before.
// ---------------------------------------------------------------------------
template <class C2>
constexpr int panel_block_smem() {   // the block, then one 32 x 32 scratch per triangle inversion
  return (LU_OUTER * LU_OUTER + 2 * SW_BLK * LU_NB * LU_NB) * (int)sizeof(C2);
}
template <class C2>
__global__ void __launch_bounds__(1024) panel_block_kernel(BatchT<C2> b, int k0, int* status) {
  extern __shared__ __align__(16) unsigned char pb_sm[];
  C2* T = reinterpret_cast<C2*>(pb_sm);   // [LU_OUTER][LU_OUTER] column-major
  C2* X = T + LU_OUTER * LU_OUTER;        // [2 * SW_BLK][LU_NB][LU_NB] inversion scratch
  const int n = b.order(blockIdx.z);
  if (k0 >= n) return;
  const int nb = min(LU_OUTER, n - k0), t = threadIdx.x;
  C2* A = b.sys(blockIdx.z);
  for (int q = t; q < LU_OUTER * LU_OUTER; q += blockDim.x) {
    const int r = q % LU_OUTER, c = q / LU_OUTER;
    T[q] = (r < nb && c < nb) ? A[(k0 + r) + (long long)n * (k0 + c)] : mkc<C2>(0., 0.);
  }
  __syncthreads();
  // thread = (row tr, every eighth column from tc0): the row's multiplier is
  // read once per step, the pivot row's entries are broadcast within a warp
  const int tr = t % LU_OUTER, tc0 = t / LU_OUTER;
  constexpr int CSTEP = 1024 / LU_OUTER;
  for (int j = 0; j < nb; ++j) {
    if (t == 0 && !(cabs2(T[j + LU_OUTER * j]) > 1.E-20)) atomicCAS(status, 0, ST_PIVOT);
    if (t > j && t < nb) T[t + LU_OUTER * j] = cdv(T[t + LU_OUTER * j], T[j + LU_OUTER * j]);
    __syncthreads();
    if (tr > j && tr < nb) {
      const C2 l = T[tr + LU_OUTER * j];
      for (int c = j + 1 + tc0; c < nb; c += CSTEP)
        T[tr + LU_OUTER * c] = cfms(T[tr + LU_OUTER * c], l, T[j + LU_OUTER * c]);
    }
    __syncthreads();
  }
  for (int q = t; q < LU_OUTER * LU_OUTER; q += blockDim.x) {
    const int r = q % LU_OUTER, c = q / LU_OUTER;
    if (r < nb && c < nb) A[(k0 + r) + (long long)n * (k0 + c)] = T[q];
  }
  // inverses of the diagonal blocks' triangles: task = (triangle, block), one
  // thread per column of the inverse; a partial last block keeps the
  // identity beyond nb (those rows and columns are never used)
  C2* P = b.pinv + (long long)blockIdx.z * PINV_SCRATCH;
  const int task = t / 128, col = t % 128;
  if (col < LU_NB) {
    const bool upper = task >= SW_BLK;
    const int bi = task % SW_BLK, o = bi * LU_NB;
    C2* x = X + task * LU_NB * LU_NB + LU_NB * col;   // this column, in shared memory
    const int nbb = max(0, min(LU_NB, nb - o));
    for (int i = 0; i < LU_NB; ++i) x[i] = mkc<C2>(i == col ? 1. : 0., 0.);
    if (col < nbb) {
      if (!upper) {   // unit lower: x_i = -sum_{k=col}^{i-1} L_ik x_k
        for (int i = col + 1; i < nbb; ++i) {
          C2 v = mkc<C2>(0., 0.);
          for (int k = col; k < i; ++k) cmac(v, T[(o + i) + LU_OUTER * (o + k)], x[k]);
          x[i] = mkc<C2>(-v.x, -v.y);
        }
      } else {        // upper: x_col = 1 / U_cc, x_i = -(sum_{k=i+1}^{col} U_ik x_k) / U_ii
        x[col] = cdv(mkc<C2>(1., 0.), T[(o + col) + LU_OUTER * (o + col)]);
        for (int i = col - 1; i >= 0; --i) {
          C2 v = mkc<C2>(0., 0.);
          for (int k = i + 1; k <= col; ++k) cmac(v, T[(o + i) + LU_OUTER * (o + k)], x[k]);
          const C2 d = cdv(v, T[(o + i) + LU_OUTER * (o + i)]);
          x[i] = mkc<C2>(-d.x, -d.y);
        }
      }
    }
    C2* dst = P + (upper ? PINV_Q_OFF : 0) + bi * LU_NB * LU_NB + LU_NB * col;
    for (int i = 0; i < LU_NB; ++i) dst[i] = x[i];
  }
}

// V = inv(U11) of the panel from the blocks of U11 (in A) and Q: column block
// j of V: V_jj = Q_jj, then for the blocks above, i = j-1 .. 0,
// V_ij = -Q_ii sum_{k=i+1}^{j} U_ik V_kj. Same layout as strip_winv_kernel.
template <class C2>
__device__ __forceinline__ void panel_vinv_body(const BatchT<C2>& b, int k0) {
  extern __shared__ __align__(16) unsigned char pv_sm[];
  constexpr int BB = LU_NB * LU_NB;
  C2* Vc = reinterpret_cast<C2*>(pv_sm);   // [SW_BLK][BB] column block j of V
  C2* S = Vc + SW_BLK * BB;
  C2* Us = S + BB;                         // U_ik (i < k) at ((k (k - 1)) / 2 + i) * BB
  C2* Qs = Us + (SW_BLK * (SW_BLK - 1) / 2) * BB;
  const int n = b.order(blockIdx.z);
  if (k0 + LU_OUTER >= n) return;
  const C2* A = b.sys(blockIdx.z);
  const C2* Q = b.pinv + (long long)blockIdx.z * PINV_SCRATCH + PINV_Q_OFF;
  C2* V = b.pinv + (long long)blockIdx.z * PINV_SCRATCH + PINV_V_OFF;
  const int r = threadIdx.x % LU_NB, c = threadIdx.x / LU_NB, e = r + LU_NB * c;
  for (int k = 1; k < SW_BLK; ++k)
    for (int i = 0; i < k; ++i)
      Us[((k * (k - 1)) / 2 + i) * BB + e] = A[(k0 + i * LU_NB + r) + (long long)n * (k0 + k * LU_NB + c)];
  for (int i = 0; i < SW_BLK; ++i) Qs[i * BB + e] = Q[i * BB + e];
  for (int j = 0; j < SW_BLK; ++j) {
    __syncthreads();
    Vc[j * BB + e] = Qs[j * BB + e];
    for (int i = j - 1; i >= 0; --i) {
      __syncthreads();   // V_kj for k > i are in shared memory
      C2 acc = mkc<C2>(0., 0.);
      for (int k = i + 1; k <= j; ++k) {
        const C2* U = Us + ((k * (k - 1)) / 2 + i) * BB + r;
        const C2* Vk = Vc + k * BB + LU_NB * c;
#pragma unroll 8
        for (int m = 0; m < LU_NB; ++m) cmac(acc, U[LU_NB * m], Vk[m]);
      }
      S[e] = acc;
      __syncthreads();
      const C2* Qi = Qs + i * BB + r;
      C2 w = mkc<C2>(0., 0.);
#pragma unroll 8
      for (int m = 0; m < LU_NB; ++m) cmac(w, Qi[LU_NB * m], S[m + LU_NB * c]);
      Vc[i * BB + e] = mkc<C2>(-w.x, -w.y);
    }
    __syncthreads();
    for (int i = 0; i <= j; ++i) V[(i * LU_NB + r) + LU_OUTER * (j * LU_NB + c)] = Vc[i * BB + e];
  }
}

// L21 = A21 V for the rows below the panel: CTA = one system and PL_R rows
// (held in shared memory, column-major, ld PL_R); thread = (row r, every
// fourth column of each 32-column block). The ten nonzero blocks of V stream
// through two shared buffers as in strip_gemm_kernel; output column block cb
// = sum_{kb <= cb} X_kb V_kb,cb.
constexpr int PL_R = 32;
template <class C2>
constexpr int panel_l21_smem() {
  return (PL_R * LU_OUTER + 2 * LU_NB * LU_NB) * (int)sizeof(C2);
}
template <class C2>
__device__ __forceinline__ void panel_l21_body(const BatchT<C2>& b, int k0, int bx) {
  extern __shared__ __align__(16) unsigned char pl_sm[];
  C2* X = reinterpret_cast<C2*>(pl_sm);   // [LU_OUTER][PL_R] the rows before the solve
  C2* Vb = X + PL_R * LU_OUTER;           // [2][LU_NB][LU_NB]
  const int n = b.order(blockIdx.z), kend = k0 + LU_OUTER;
  const int r0 = kend + bx * PL_R, nrow = min(PL_R, n - r0);
  if (nrow <= 0) return;
  C2* A = b.sys(blockIdx.z);
  const C2* V = b.pinv + (long long)blockIdx.z * PINV_SCRATCH + PINV_V_OFF;
  // block step s -> (kb, cb) with kb <= cb: (0,0), (0,1), (1,1), (0,2), ...
  auto blk = [](int s, int& kb, int& cb) {
    cb = 0;
    while ((cb + 1) * (cb + 2) / 2 <= s) ++cb;
    kb = s - cb * (cb + 1) / 2;
  };
  auto fetch = [&](int s) {
    int kb, cb;
    blk(s, kb, cb);
    C2* dst = Vb + (s & 1) * LU_NB * LU_NB;
    for (int q = threadIdx.x; q < LU_NB * LU_NB; q += blockDim.x) {
      const int rr = q % LU_NB, cc = q / LU_NB;
      cp_async_elem(dst + q, V + (kb * LU_NB + rr) + LU_OUTER * (cb * LU_NB + cc), true);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  fetch(0);
  for (int q = threadIdx.x; q < PL_R * LU_OUTER; q += blockDim.x) {
    const int rr = q % PL_R, cc = q / PL_R;
    X[q] = rr < nrow ? A[(r0 + rr) + (long long)n * (k0 + cc)] : mkc<C2>(0., 0.);
  }
  const int r = threadIdx.x % PL_R, g = threadIdx.x / PL_R;
  constexpr int GROUPS = 128 / PL_R, CPT = LU_NB / GROUPS, NSTEP = SW_BLK * (SW_BLK + 1) / 2;
  C2 acc[CPT];
  for (int s = 0; s < NSTEP; ++s) {
    int kb, cb;
    blk(s, kb, cb);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    if (s + 1 < NSTEP) fetch(s + 1);
    if (kb == 0) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) acc[m] = mkc<C2>(0., 0.);
    }
    const C2* Vt = Vb + (s & 1) * LU_NB * LU_NB;
    for (int j = 0; j < LU_NB; j += 2) {   // two k at a time: one 16-byte load gives both V entries
      const C2 x0 = X[(kb * LU_NB + j) * PL_R + r], x1 = X[(kb * LU_NB + j + 1) * PL_R + r];
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        C2 v0, v1;
        ld_pair(Vt + j + LU_NB * (g + GROUPS * m), v0, v1);
        cmac(acc[m], x0, v0);
        cmac(acc[m], x1, v1);
      }
    }
    if (kb == cb && r < nrow) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) A[(r0 + r) + (long long)n * (k0 + cb * LU_NB + g + GROUPS * m)] = acc[m];
    }
  }
}

template <class C2>
__global__ void __launch_bounds__(LU_NB * LU_NB) strip_winv_kernel(BatchT<C2> b, int k0) {
  strip_winv_body(b, k0);
}
template <class C2>
__global__ void __launch_bounds__(128) strip_gemm_kernel(BatchT<C2> b, int k0) {
  strip_gemm_body(b, k0, blockIdx.x);
}
// both triangle inverses of the panel's diagonal block: blockIdx.x 0 W, 1 V
template <class C2>
__global__ void __launch_bounds__(LU_NB * LU_NB) panel_inv_kernel(BatchT<C2> b, int k0) {
  if (blockIdx.x == 0) strip_winv_body(b, k0);
  else panel_vinv_body(b, k0);
}
// both block products of the panel: blockIdx.y 0 L21 = A21 V (row chunks),
// 1 U12 = W A12 (column chunks)
template <class C2>
constexpr int panel_products_smem() {
  return panel_l21_smem<C2>() > strip_gemm_smem<C2>() ? panel_l21_smem<C2>() : strip_gemm_smem<C2>();
}
template <class C2>
__global__ void __launch_bounds__(128) panel_products_kernel(BatchT<C2> b, int k0) {
  if (blockIdx.y == 0) panel_l21_body(b, k0, blockIdx.x);
  else strip_gemm_body(b, k0, blockIdx.x);
}

// Systems split into groups factored side by side on separate streams: the
// launches of a step are issued group after group, so the latency-bound
// kernels of one group (diagonal blocks, panels, small updates) overlap the
// work of the other. Without lanes (or with one system) everything runs on
// the caller's stream.
#ifndef NB_LANES
#define NB_LANES 4
#endif
constexpr int LANES = NB_LANES;
struct Lanes {
  cudaStream_t s[LANES] = {};
  cudaEvent_t fork = nullptr, join[LANES] = {};
};

struct LaneSplit {
  int groups = 1;
  int first[LANES + 1] = {};
  cudaStream_t st[LANES] = {};
};

// FP32 panels factored as one block per system (default), or by LU_NB-column
// steps with NEMOH_B200_PANEL=steps
inline bool panel_as_block() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_PANEL");
    return !(e && std::strcmp(e, "steps") == 0);
  }();
  return on;
}

// row strips as W = inv(L11) times the strip (default), or by the blocked
// forward solve with NEMOH_B200_STRIP=solve
inline bool strip_as_product() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_STRIP");
    return !(e && std::strcmp(e, "solve") == 0);
  }();
  return on;
}

// stream groups in use: LANES, or fewer with NEMOH_B200_LANES (1..LANES)
inline int lane_count() {
  static const int n = [] {
    const char* e = std::getenv("NEMOH_B200_LANES");
    const int v = e ? std::atoi(e) : LANES;
    return std::max(1, std::min(LANES, v));
  }();
  return n;
}

inline LaneSplit lane_split(int nsys, cudaStream_t main, const Lanes* lanes) {
  LaneSplit L;
  if (!lanes || !lanes->s[0] || nsys < 2 || lane_count() < 2) {   // one group: the caller's stream
    L.groups = 1;
    L.first[0] = 0;
    L.first[1] = nsys;
    L.st[0] = main;
    return L;
  }
  L.groups = std::min(lane_count(), nsys);   // every group holds at least one system
  for (int g = 0; g <= L.groups; ++g) L.first[g] = (int)((long long)nsys * g / L.groups);
  cudaEventRecord(lanes->fork, main);
  for (int g = 0; g < L.groups; ++g) {
    L.st[g] = lanes->s[g];
    cudaStreamWaitEvent(lanes->s[g], lanes->fork, 0);
  }
  return L;
}

inline void lane_join(const LaneSplit& L, cudaStream_t main, const Lanes* lanes) {
  if (L.groups == 1) return;
  for (int g = 0; g < L.groups; ++g) {
    cudaEventRecord(lanes->join[g], L.st[g]);
    cudaStreamWaitEvent(main, lanes->join[g], 0);
  }
}

template <class C2>
inline BatchT<C2> sub_batch(const BatchT<C2>& b, int s0) {
  BatchT<C2> r = b;
  if (b.off) {
    r.off = b.off + s0;
    r.ord = b.ord + s0;
  } else {
    r.base = b.base + s0 * b.stride;
  }
  r.diag = b.diag + (long long)s0 * DIAG_SCRATCH;
  if (b.pinv) r.pinv = b.pinv + (long long)s0 * PINV_SCRATCH;
  return r;
}

// outer(bsub, nsub, stream, s0, k0, kend): trailing update of one group.
// host_ord (ragged batches): the systems' orders on the host, in decreasing
// order; at every step only the systems still above it are launched (a prefix
// of each group) and the grids are sized by the group's largest system.
template <class C2, class Outer>
inline void lu_two_level(BatchT<C2> b, int nsys, int* status, cudaStream_t main, long long& launches, Outer outer,
                         const Lanes* lanes = nullptr, const int* host_ord = nullptr, bool outer_products = false) {
  const int n = b.n;
  const LaneSplit L = lane_split(nsys, main, lanes);
  // NEMOH_B200_OUTER_JOIN=1: the groups join for each outer update, which
  // then covers every system in one launch
  static const bool join_env = [] {
    const char* e = std::getenv("NEMOH_B200_OUTER_JOIN");
    return e && e[0] == '1';
  }();
  const bool join_outer = join_env && L.groups > 1;
  // systems of group g whose order exceeds k
  auto active = [&](int g, int k) {
    const int s0 = L.first[g], s1 = L.first[g + 1];
    if (!host_ord) return k < n ? s1 - s0 : 0;
    int c = 0;
    while (s0 + c < s1 && host_ord[s0 + c] > k) ++c;
    return c;
  };
  // the FP32 row-strip form factors each panel as one block (panel_block_kernel)
  const bool block = b.pinv && sizeof(C2) == sizeof(float2) && panel_as_block();
  if (block) {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
      cudaFuncSetAttribute(panel_block_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           panel_block_smem<C2>());
      cudaFuncSetAttribute(panel_inv_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, strip_winv_smem<C2>());
      cudaFuncSetAttribute(panel_products_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           panel_products_smem<C2>());
    });
  }
  for (int k0 = 0; k0 < n; k0 += LU_OUTER) {
    if (block) {
      for (int g = 0; g < L.groups; ++g) {
        const int ns = active(g, k0);
        if (ns == 0) continue;
        const int s0 = L.first[g];
        const int ng = host_ord ? host_ord[s0] : n;
        const int kend = std::min(k0 + LU_OUTER, ng);
        BatchT<C2> bg = sub_batch(b, s0);
        bg.n = ng;
        const cudaStream_t st = L.st[g];
        panel_block_kernel<C2><<<dim3(1, 1, ns), 1024, panel_block_smem<C2>(), st>>>(bg, k0, status);
        ++launches;
        if (kend >= ng) continue;
        panel_inv_kernel<C2><<<dim3(2, 1, ns), LU_NB * LU_NB, strip_winv_smem<C2>(), st>>>(bg, k0);
        ++launches;
        if (!outer_products) {   // else outer() forms L21 and U12 (on the tensor cores) before its update
          const int nx = std::max((ng - kend + PL_R - 1) / PL_R, (ng - kend + ST_C - 1) / ST_C);
          panel_products_kernel<C2><<<dim3(nx, 2, ns), 128, panel_products_smem<C2>(), st>>>(bg, k0);
          ++launches;
        }
        if (!join_outer) outer(bg, ns, st, s0, k0, kend);
      }
      if (join_outer) {
        const int ng = host_ord ? host_ord[0] : n;
        const int kend = std::min(k0 + LU_OUTER, ng);
        int ns = 0;
        for (int g = 0; g < L.groups; ++g) ns = std::max(ns, L.first[g] + active(g, k0));
        if (kend < ng && ns > 0) {
          lane_join(L, main, lanes);
          BatchT<C2> bw = b;
          bw.n = ng;
          outer(bw, ns, main, 0, k0, kend);
          cudaEventRecord(lanes->fork, main);
          for (int g = 0; g < L.groups; ++g) cudaStreamWaitEvent(L.st[g], lanes->fork, 0);
        }
      }
      continue;
    }
    for (int k = k0; k < std::min(k0 + LU_OUTER, n); k += LU_NB) {
      for (int g = 0; g < L.groups; ++g) {
        const int ns = active(g, k);
        if (ns == 0) continue;
        const int s0 = L.first[g];
        const int ng = host_ord ? host_ord[s0] : n;   // largest order in the group
        const int kend = std::min(k0 + LU_OUTER, ng);
        const int nb = std::min(LU_NB, ng - k), rest = ng - k - nb;
        const int nrb = (rest + LU_RB - 1) / LU_RB;
        // with b.pinv the row strip right of the panel waits for strip_kernel
        const int ucol = b.pinv ? kend : ng;
        const int ncb_used = (std::max(0, ucol - k - nb) + LU_CB - 1) / LU_CB;
        BatchT<C2> bg = sub_batch(b, s0);
        bg.n = ng;
        const cudaStream_t st = L.st[g];
        lu_diag_kernel<C2><<<dim3(1, 1, ns), LU_DIAG_THREADS, 0, st>>>(bg, k, status);
        ++launches;
        lu_panel_kernel<C2><<<dim3(std::max(1, nrb + ncb_used), 1, ns), LU_RB, 0, st>>>(bg, k, ucol);
        ++launches;
        if (k + nb < kend) {
          zgemm_update<C2>(bg, k, nb, Rect{k + nb, ng, k + nb, kend}, ns, st);
          ++launches;
          if (kend < ng && !b.pinv) {
            zgemm_update<C2>(bg, k, nb, Rect{k + nb, kend, kend, ng}, ns, st);
            ++launches;
          }
        }
      }
    }
    for (int g = 0; g < L.groups; ++g) {
      const int ns = active(g, k0);
      if (ns == 0) continue;
      const int s0 = L.first[g];
      const int ng = host_ord ? host_ord[s0] : n;
      const int kend = std::min(k0 + LU_OUTER, ng);
      if (kend >= ng) continue;
      BatchT<C2> bg = sub_batch(b, s0);
      bg.n = ng;
      const cudaStream_t st = L.st[g];
      if (b.pinv) {
        static std::atomic<unsigned long long> attr{0};
        once_per_device(attr, [] {
          cudaFuncSetAttribute(strip_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, strip_smem<C2>());
          cudaFuncSetAttribute(strip_winv_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               strip_winv_smem<C2>());
          cudaFuncSetAttribute(strip_gemm_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               strip_gemm_smem<C2>());
        });
        const dim3 sgrid((ng - kend + ST_C - 1) / ST_C, 1, ns);
        if (strip_as_product()) {
          strip_winv_kernel<C2><<<dim3(1, 1, ns), LU_NB * LU_NB, strip_winv_smem<C2>(), st>>>(bg, k0);
          strip_gemm_kernel<C2><<<sgrid, 128, strip_gemm_smem<C2>(), st>>>(bg, k0);
          launches += 2;
        } else {
          strip_kernel<C2><<<sgrid, 128, strip_smem<C2>(), st>>>(bg, k0);
          ++launches;
        }
      }
      if (!join_outer) outer(bg, ns, st, s0, k0, kend);
    }
    if (join_outer) {   // one trailing update for every group, then the groups go on
      const int ng = host_ord ? host_ord[0] : n;
      const int kend = std::min(k0 + LU_OUTER, ng);
      int ns = 0;
      for (int g = 0; g < L.groups; ++g) ns = std::max(ns, L.first[g] + active(g, k0));
      if (kend < ng && ns > 0) {
        lane_join(L, main, lanes);
        BatchT<C2> bw = b;
        bw.n = ng;
        outer(bw, ns, main, 0, k0, kend);
        cudaEventRecord(lanes->fork, main);
        for (int g = 0; g < L.groups; ++g) cudaStreamWaitEvent(L.st[g], lanes->fork, 0);
      }
    }
  }
  lane_join(L, main, lanes);
}

constexpr int MAX_RHS = 16;

// B = (NVEL(I) +- NVEL(I+NFA))/2 per symmetry class (SOLVE_BEM_INFD_DIRECT.f90:123-131)
// nvel: (2^s n) x nrhs per frequency; X: system (w, class) at (w*cls+class)*n*nrhs
__global__ void fold_rhs_kernel(const double2* __restrict__ nvel, int n, int nsymy, int nrhs, double2* __restrict__ X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = blockIdx.y, w = blockIdx.z;
  const int cls = nsymy ? 2 : 1;
  const double2* v = nvel + ((long long)w * nrhs + p) * cls * n;
  if (nsymy) {
    const double2 a = v[i], b = v[i + n];
    X[((long long)w * 2 + 0) * n * nrhs + (long long)p * n + i] = make_double2((a.x + b.x) * 0.5, (a.y + b.y) * 0.5);
    X[((long long)w * 2 + 1) * n * nrhs + (long long)p * n + i] = make_double2((a.x - b.x) * 0.5, (a.y - b.y) * 0.5);
  } else {
    X[(long long)w * n * nrhs + (long long)p * n + i] = v[i];
  }
}

// One (body, frequency) item of a ragged batch: where its inputs and outputs
// are in the caller's arrays (items in the caller's order) and where its
// systems are in the batch (sorted by decreasing order).
struct ItemDesc {
  long long nvel_off;    // complex offset of the item's NVEL, (2^s n) x nrhs column-major
  long long force_off;   // complex offset of the item's forces, nint x nrhs
  const double* nds;     // the body's generalised normals, nint x (2^s n)
  double rho;
  int n, nsymy, sys0, nint;
};

// fold_rhs_kernel per item; X: system s at s * xstride, leading dimension n
__global__ void fold_rhs_ragged_kernel(const double2* __restrict__ nvel, const ItemDesc* __restrict__ items, int nrhs,
                                       long long xstride, double2* __restrict__ X) {
  const ItemDesc it = items[blockIdx.z];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, p = blockIdx.y, n = it.n;
  if (i >= n) return;
  const int cls = it.nsymy ? 2 : 1;
  const double2* v = nvel + it.nvel_off + (long long)p * cls * n;
  double2* x0 = X + it.sys0 * xstride + (long long)p * n;
  if (it.nsymy) {
    const double2 a = v[i], b = v[i + n];
    x0[i] = make_double2((a.x + b.x) * 0.5, (a.y + b.y) * 0.5);
    x0[xstride + i] = make_double2((a.x - b.x) * 0.5, (a.y - b.y) * 0.5);
  } else {
    x0[i] = v[i];
  }
}

// force_kernel per item (its frequency's parameters in oms[item])
__global__ void __launch_bounds__(256) force_ragged_kernel(const double2* __restrict__ phi,
                                                           const ItemDesc* __restrict__ items,
                                                           const OmegaParams* __restrict__ oms, int nrhs,
                                                           long long xstride, double2* __restrict__ force) {
  const ItemDesc it = items[blockIdx.z];
  const int i = blockIdx.x, p = blockIdx.y, n = it.n;
  if (i >= it.nint) return;
  const int cls = it.nsymy ? 2 : 1;
  const double2* pp = phi + it.sys0 * xstride + (long long)p * n;
  const double2* pm = pp + (cls - 1) * xstride;
  double sr = 0., si = 0.;
  for (int c = threadIdx.x; c < cls * n; c += blockDim.x) {
    double2 z;
    if (!it.nsymy) z = pp[c];
    else if (c < n) z = make_double2(pp[c].x + pm[c].x, pp[c].y + pm[c].y);
    else z = make_double2(pp[c - n].x - pm[c - n].x, pp[c - n].y - pm[c - n].y);
    const double f = it.nds[i + (long long)it.nint * c];
    sr += z.x * f;
    si += z.y * f;
  }
  __shared__ double red[2][256];
  red[0][threadIdx.x] = sr;
  red[1][threadIdx.x] = si;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rw = it.rho * oms[blockIdx.z].w;
    force[it.force_off + (long long)p * it.nint + i] = make_double2(rw * red[1][0], -rw * red[0][0]);
  }
}

// Force(i,p) = -sum_c PRESSURE(c) NDS(i,c), PRESSURE = RHO*i*W*ZP with
// ZP = phi+ + phi- on the meshed half and phi+ - phi- on its mirror
// (SOLVE_BEM.f90:91-96, NEMOH.f90:137-141). phi: system (w,class) n x nrhs.
__global__ void __launch_bounds__(256) force_kernel(const double2* __restrict__ phi, const OmegaParams* __restrict__ oms,
                                                    int n, int nsymy, int nrhs, int nint, const double* __restrict__ nds,
                                                    double rho, double2* __restrict__ force) {
  const int i = blockIdx.x, p = blockIdx.y, w = blockIdx.z;
  const int cls = nsymy ? 2 : 1;
  const double2* pp = phi + ((long long)w * cls + 0) * n * nrhs + (long long)p * n;
  const double2* pm = phi + ((long long)w * cls + (cls - 1)) * n * nrhs + (long long)p * n;
  double sr = 0., si = 0.;
  for (int c = threadIdx.x; c < cls * n; c += blockDim.x) {
    double2 z;
    if (!nsymy) z = pp[c];
    else if (c < n) z = make_double2(pp[c].x + pm[c].x, pp[c].y + pm[c].y);
    else z = make_double2(pp[c - n].x - pm[c - n].x, pp[c - n].y - pm[c - n].y);
    const double f = nds[i + (long long)nint * c];
    sr += z.x * f;
    si += z.y * f;
  }
  __shared__ double red[2][256];
  red[0][threadIdx.x] = sr;
  red[1][threadIdx.x] = si;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rw = rho * oms[w].w;
    // -(i rho W) * sum(ZP * NDS)
    force[((long long)w * nrhs + p) * nint + i] = make_double2(rw * red[1][0], -rw * red[0][0]);
  }
}


// ---------------------------------------------------------------------------
// Blocked triangular solves with precomputed inverses of the diagonal blocks.
// After the factorization, inv_diag_kernel stores inv(L_bb) and inv(U_bb) for
// every TB x TB diagonal block; a solve step is then a small block product
// x_b = inv(T_bb) r_b plus the update of the remaining rows.
// ---------------------------------------------------------------------------
constexpr int TB = 64;
constexpr int TRSM_ROWS = 32;   // rows updated per CTA of a solve step

template <class C2>
__device__ __forceinline__ void cmad(C2& acc, C2 a, C2 b) {
  cmac(acc, a, b);
}

// inv layout: ((sys * nblk + blk) * 2 + {0: inv L, 1: inv U}) * TB * TB, column-major.
// Inverses of the unit-lower and upper triangles of the TB x TB diagonal
// blocks (a partial last block is padded with the identity): 1024 threads, each
// owning row i of four columns, one barrier per elimination step. inv(L):
// X = I, step j (ascending) subtracts L(i, j) X(j, :) from the rows below
// (the order of the column-by-column forward substitution); inv(U): X = I, step
// j (descending) divides row j by U(j, j), then subtracts U(i, j) X(j, :) from
// the rows above.
constexpr int INV_THREADS = 1024;
template <class C2>
constexpr int inv_diag_smem() {
  return 3 * TB * TB * (int)sizeof(C2);
}
template <class C2>
__global__ void __launch_bounds__(INV_THREADS) inv_diag_kernel(BatchT<C2> b, C2* __restrict__ inv, int nblk) {
  extern __shared__ __align__(16) unsigned char dsm[];
  C2* T = reinterpret_cast<C2*>(dsm);   // [TB][TB] the block
  C2* XL = T + TB * TB;                 // inv(L)
  C2* XU = XL + TB * TB;                // inv(U)
  const int n = b.order(blockIdx.z), blk = blockIdx.x, k = blk * TB, nb = min(TB, n - k);
  if (nb <= 0) return;
  const C2* A = b.sys(blockIdx.z);
  const C2 one = mkc<C2>(1., 0.), zero = mkc<C2>(0., 0.);
  for (int q = threadIdx.x; q < TB * TB; q += blockDim.x) {
    const int i = q % TB, c = q / TB;
    T[q] = (i < nb && c < nb) ? A[(k + i) + (long long)n * (k + c)] : (i == c ? one : zero);
    XL[q] = i == c ? one : zero;
    XU[q] = i == c ? one : zero;
  }
  __syncthreads();
  constexpr int CG = INV_THREADS / TB;   // column groups: columns cq + CG m
  const int i = threadIdx.x % TB, cq = threadIdx.x / TB;
  for (int step = 0; step < TB; ++step) {
    const int jl = step, ju = TB - 1 - step;
    if (i == ju)
#pragma unroll
      for (int m = 0; m < TB / CG; ++m) {
        const int c = cq + CG * m;
        if (c >= ju) XU[ju + TB * c] = cdv(XU[ju + TB * c], T[ju + TB * ju]);
      }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < TB / CG; ++m) {
      const int c = cq + CG * m;
      if (i > jl && c <= jl) XL[i + TB * c] = cfms(XL[i + TB * c], T[i + TB * jl], XL[jl + TB * c]);
      if (i < ju && c >= ju) XU[i + TB * c] = cfms(XU[i + TB * c], T[i + TB * ju], XU[ju + TB * c]);
    }
    __syncthreads();
  }
  C2* out = inv + ((long long)(blockIdx.z * nblk + blk) * 2) * TB * TB;
  for (int q = threadIdx.x; q < TB * TB; q += blockDim.x) {
    out[q] = XL[q];
    out[TB * TB + q] = XU[q];
  }
}

// Triangular solves, one launch per diagonal block. X holds the running
// right-hand sides, Y receives the solution. A launch for block b applies the
// solved block (already in Y) to the rows still to come, 64 rows per CTA;
// the CTA holding block b+1 (forward) or b-1 (backward) then solves it with
// the inverted diagonal block and stores it in Y for the next launch.
// With apply = false the launch only solves block b (the first step).
template <class C2, bool LOWER>
__global__ void __launch_bounds__(128) trsm_fused_kernel(BatchT<C2> b, const C2* __restrict__ inv, int nblk, C2* xbase,
                                                         C2* ybase, long long xstride, int nrhs, int blk, int apply) {
  extern __shared__ __align__(16) unsigned char dsm[];
  C2* Sb = reinterpret_cast<C2*>(dsm);   // [TB][MAX_RHS] solved block blk
  C2* Xn = Sb + TB * MAX_RHS;            // [TB][MAX_RHS] next block, updated
  C2* Ti = Xn + TB * MAX_RHS;            // [TB][TB] inverse of the next diagonal block
  const int n = b.n;
  const C2* A = b.base + blockIdx.z * b.stride;
  C2* X = xbase + blockIdx.z * xstride;
  C2* Y = ybase + blockIdx.z * xstride;
  int nxt = blk;            // block solved by CTA 0 at the end
  // CTA 0 starts copying the inverse of the block it will solve while it
  // still applies the previous block
  const int solve_blk = apply ? (LOWER ? blk + 1 : blk - 1) : blk;
  const bool solver = blockIdx.x == 0 && solve_blk >= 0 && solve_blk < nblk;
  if (solver) {
    const C2* src = inv + ((long long)(blockIdx.z * nblk + solve_blk) * 2 + (LOWER ? 0 : 1)) * TB * TB;
    for (int q = threadIdx.x; q < TB * TB; q += blockDim.x) cp_async_elem(Ti + q, src + q, true);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  if (apply) {
    const int k = blk * TB, nb = min(TB, n - k);
    for (int q = threadIdx.x; q < TB * nrhs; q += blockDim.x) {
      const int i = q % TB, p = q / TB;
      Sb[i + TB * p] = (i < nb) ? Y[(k + i) + (long long)n * p] : mkc<C2>(0., 0.);
    }
    __syncthreads();
    // rows of this CTA: forward [k+nb+64c, ...), backward [k-64(c+1), k-64c).
    // A lane pair shares a row: lane parity picks the half of the 64 columns,
    // and the two partial sums meet through a shuffle.
    const int r0 = LOWER ? k + nb + (int)blockIdx.x * TB : k - ((int)blockIdx.x + 1) * TB;
    const int row = threadIdx.x >> 1, part = threadIdx.x & 1;
    const int r = r0 + row;
    const bool live = LOWER ? (r < n) : (r >= 0);
    C2 a[TB / 2];
#pragma unroll
    for (int j = 0; j < TB / 2; ++j) {
      const int c = part * (TB / 2) + j;
      a[j] = (live && c < nb) ? A[r + (long long)n * (k + c)] : mkc<C2>(0., 0.);
    }
    const C2* Sp = Sb + part * (TB / 2);
    for (int p = 0; p < nrhs; ++p) {
      C2 acc = mkc<C2>(0., 0.);
#pragma unroll
      for (int j = 0; j < TB / 2; ++j) cmad(acc, a[j], Sp[j + TB * p]);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      if (part == 0 && live) {
        C2* q = X + r + (long long)n * p;
        C2 v = *q;
        v.x -= acc.x;
        v.y -= acc.y;
        *q = v;
        if (blockIdx.x == 0) Xn[row + TB * p] = v;
      }
    }
    __syncthreads();
    if (blockIdx.x != 0) return;
    nxt = LOWER ? blk + 1 : blk - 1;
    if (nxt < 0 || nxt >= nblk) return;
  } else {
    if (blockIdx.x != 0) return;
    const int k = nxt * TB, nb = min(TB, n - k);
    for (int q = threadIdx.x; q < TB * nrhs; q += blockDim.x) {
      const int i = q % TB, p = q / TB;
      Xn[i + TB * p] = (i < nb) ? X[(k + i) + (long long)n * p] : mkc<C2>(0., 0.);
    }
  }
  // CTA 0: solve block nxt from Xn (rows beyond n are zero)
  const int kn = nxt * TB, nbn = min(TB, n - kn);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (apply)
    for (int q = threadIdx.x; q < TB * nrhs; q += blockDim.x) {
      const int i = q % TB, p = q / TB;
      if (i >= nbn) Xn[i + TB * p] = mkc<C2>(0., 0.);
    }
  __syncthreads();
  for (int q = threadIdx.x; q < nbn * nrhs; q += blockDim.x) {
    const int i = q % nbn, p = q / nbn;
    C2 acc = mkc<C2>(0., 0.);
    for (int j = 0; j < TB; ++j) cmad(acc, Ti[i + TB * j], Xn[j + TB * p]);
    Y[(kn + i) + (long long)n * p] = acc;
  }
}

// Forward then backward solve of the factored systems: X holds the right-hand
// sides and receives the solution, Y is scratch of the same size.
template <class C2>
void trsm_launch(BatchT<C2> b, const C2* inv, C2* X, C2* Y, int nsys, int nrhs, cudaStream_t main, long long& launches,
                 const Lanes* lanes = nullptr) {
  const int N = b.n;
  const long long xs = (long long)N * nrhs;
  const int nblk = (N + TB - 1) / TB;
  const int smem = (2 * TB * MAX_RHS + TB * TB) * (int)sizeof(C2);
  static std::atomic<unsigned long long> attr{0};
  once_per_device(attr, [smem] {
    cudaFuncSetAttribute(trsm_fused_kernel<C2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(trsm_fused_kernel<C2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
  const LaneSplit L = lane_split(nsys, main, lanes);
  auto each = [&](auto launch) {
    for (int g = 0; g < L.groups; ++g) {
      const int s0 = L.first[g], ns = L.first[g + 1] - s0;
      BatchT<C2> bg = b;
      bg.base = b.base + s0 * b.stride;
      launch(bg, inv + (long long)s0 * nblk * 2 * TB * TB, X + s0 * xs, Y + s0 * xs, ns, L.st[g]);
    }
  };
  // forward: X -> Y
  each([&](BatchT<C2> bg, const C2* ig, C2* xg, C2* yg, int ns, cudaStream_t st) {
    trsm_fused_kernel<C2, true><<<dim3(1, 1, ns), 128, smem, st>>>(bg, ig, nblk, xg, yg, xs, nrhs, 0, 0);
    ++launches;
  });
  for (int blk = 0; blk + 1 < nblk; ++blk) {
    const int below = N - std::min(N, (blk + 1) * TB);
    each([&](BatchT<C2> bg, const C2* ig, C2* xg, C2* yg, int ns, cudaStream_t st) {
      trsm_fused_kernel<C2, true><<<dim3(std::max(1, (below + TB - 1) / TB), 1, ns), 128, smem, st>>>(
          bg, ig, nblk, xg, yg, xs, nrhs, blk, 1);
      ++launches;
    });
  }
  // backward: Y -> X
  each([&](BatchT<C2> bg, const C2* ig, C2* xg, C2* yg, int ns, cudaStream_t st) {
    trsm_fused_kernel<C2, false><<<dim3(1, 1, ns), 128, smem, st>>>(bg, ig, nblk, yg, xg, xs, nrhs, nblk - 1, 0);
    ++launches;
  });
  for (int blk = nblk - 1; blk >= 1; --blk) {
    each([&](BatchT<C2> bg, const C2* ig, C2* xg, C2* yg, int ns, cudaStream_t st) {
      trsm_fused_kernel<C2, false><<<dim3(blk, 1, ns), 128, smem, st>>>(bg, ig, nblk, yg, xg, xs, nrhs, blk, 1);
      ++launches;
    });
  }
  lane_join(L, main, lanes);
}

// ---------------------------------------------------------------------------
// Triangular sweep in one launch per direction. A thread-block cluster of
// `csize` CTAs (1..8, one cluster per system along grid.x) owns the 64-row
// blocks of one system cyclically (block i belongs to CTA i mod csize). Step s
// of the forward sweep:
//   * every CTA copies the solved block y_s from its owner's shared memory
//     (distributed shared memory) and subtracts L[rows, block s] y_s from the
//     right-hand sides of its own rows below block s (right-looking, so a row
//     block only ever receives updates from the CTA that owns it);
//   * the owner of block s+1, whose rows are then complete, solves
//     y_{s+1} = inv(L_{s+1,s+1}) r_{s+1} with the inverted diagonal block
//     (prefetched by cp.async during the update) into one of two shared
//     buffers, and writes it to Y;
//   * one cluster barrier (hardware) ends the step. The two y buffers
//     alternate, so a buffer is rewritten only after the barrier that follows
//     every read of it.
// The backward sweep runs the same way from the last block with U. X holds the
// right-hand sides and is overwritten by partial sums; Y receives the solution.
// `active` (may be null): refinement flags, [0] for the whole launch (it
// does nothing when 0: a converged refinement) and [1 + s] for system s
// (its cluster leaves at once when 0: that system has converged).
// ---------------------------------------------------------------------------
constexpr int SW_THREADS = 256;
template <class C2, int NR>
constexpr int sweep_smem() {
  return (TB * TB + 4 * TB * NR) * (int)sizeof(C2);   // inverse block, y buffers x2, local y, r block
}

template <class C2, int NR, bool LOWER>
__global__ void __launch_bounds__(SW_THREADS, sizeof(C2) == sizeof(float2) ? 2 : 1)
    trsm_sweep_kernel(BatchT<C2> b, const C2* __restrict__ inv, int nblk,
                                                                C2* xbase, C2* ybase, long long xstride,
                                                                const int* active) {
  namespace cg = cooperative_groups;
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char sw_sm[];
  C2* Ti = reinterpret_cast<C2*>(sw_sm);   // [TB][TB] inverse of the block being solved, column-major
  C2* ybuf = Ti + TB * TB;                 // [2][NR][TB] solved blocks (read by the whole cluster)
  C2* yloc = ybuf + 2 * TB * NR;           // [NR][TB] local copy of the block applied in this step
  C2* rb = yloc + TB * NR;                 // [NR][TB] right-hand sides of the block being solved
  cg::cluster_group cl = cg::this_cluster();
  const int csize = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int sys = blockIdx.x / csize;
  if (active && active[1 + sys] == 0) return;   // this system has converged (whole cluster)
  const int n = b.order(sys);
  const C2* A = b.sys(sys);
  C2* X = xbase + sys * xstride;
  C2* Y = ybase + sys * xstride;
  // nblk: the stride of the inverted blocks per system; this system has nbs blocks
  const C2* invs = inv + (long long)sys * nblk * 2 * TB * TB + (LOWER ? 0 : TB * TB);
  const int nbs = (n + TB - 1) / TB;
  const int t = threadIdx.x;
  const int step = LOWER ? 1 : -1;
  const int first = LOWER ? 0 : nbs - 1, last = LOWER ? nbs - 1 : 0;
  auto prefetch_inv = [&](int blk) {
    const C2* src = invs + (long long)blk * 2 * TB * TB;
    for (int q = t; q < TB * TB; q += SW_THREADS) cp_async_elem(Ti + q, src + q, true);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // owner: rb <- X rows of blk (zero past n), then y = Ti rb into ybuf[blk & 1] and Y
  auto solve = [&](int blk) {
    const int k = blk * TB, nb = min(TB, n - k);
    for (int q = t; q < TB * NR; q += SW_THREADS) {
      const int i = q % TB, p = q / TB;
      rb[q] = i < nb ? X[(k + i) + (long long)n * p] : mkc<C2>(0., 0.);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    C2* yb = ybuf + (blk & 1) * TB * NR;
    const int i = t % TB;
    for (int p = t / TB; p < NR; p += SW_THREADS / TB) {
      C2 acc = mkc<C2>(0., 0.);
#pragma unroll 8
      for (int j = 0; j < TB; ++j) cmac(acc, Ti[i + TB * j], rb[j + TB * p]);
      yb[i + TB * p] = acc;
      if (i < nb) Y[(k + i) + (long long)n * p] = acc;
    }
  };
  if (rank == first % csize) {
    prefetch_inv(first);
    solve(first);
  }
  cl.sync();
  for (int s = first; s != last; s += step) {
    const int nxt = s + step;
    const bool owns_next = rank == nxt % csize;
    if (owns_next) prefetch_inv(nxt);
    const C2* src = cl.map_shared_rank(ybuf + (s & 1) * TB * NR, s % csize);
    for (int q = t; q < TB * NR; q += SW_THREADS) yloc[q] = src[q];
    __syncthreads();
    // own row blocks still to come: forward i > s, backward i < s
    const int k = s * TB, nb = min(TB, n - k);
    const int i0 = LOWER ? s + 1 : 0, i1 = LOWER ? nbs : s;   // [i0, i1)
    int mine0 = i0 + ((rank - i0 % csize) % csize + csize) % csize;   // first block >= i0 owned here
    for (int ib = mine0 + (t / TB) * csize; ib < i1; ib += (SW_THREADS / TB) * csize) {
      const int r = ib * TB + (t % TB);
      if (r >= n) continue;
      const C2* Ar = A + r + (long long)n * k;
      C2 acc[NR];
#pragma unroll
      for (int p = 0; p < NR; ++p) acc[p] = mkc<C2>(0., 0.);
      // the row's columns of block s are loaded 32 (FP32; two CTAs of 256
      // threads fit an SM) or 16 (FP64) at a time before any is used, so a
      // thread keeps that many loads in flight
      constexpr int PF = sizeof(C2) == sizeof(float2) ? 32 : 16;
      C2 a[PF];
#pragma unroll 1
      for (int c0 = 0; c0 < nb; c0 += PF) {
#pragma unroll
        for (int j = 0; j < PF; ++j) a[j] = (c0 + j < nb) ? Ar[(long long)n * (c0 + j)] : mkc<C2>(0., 0.);
#pragma unroll
        for (int j = 0; j < PF; ++j)
#pragma unroll
          for (int p = 0; p < NR; ++p) cmac(acc[p], a[j], yloc[(c0 + j) + TB * p]);
      }
#pragma unroll
      for (int p = 0; p < NR; ++p) {
        C2* q = X + r + (long long)n * p;
        C2 v = *q;
        v.x -= acc[p].x;
        v.y -= acc[p].y;
        *q = v;
      }
    }
    __syncthreads();
    if (owns_next) solve(nxt);
    cl.sync();
  }
}

// cluster size of the sweep: enough CTAs in flight for the device (about two
// per SM), at most 8 per system (portable cluster size), a power of two
inline int sweep_cluster(int nsys, int nblk, int sms) {
  int c = 1;
  while (c < 8 && c < nblk && (long long)nsys * c < 2LL * sms) c *= 2;
  return c;
}

template <class C2, int NR, bool LOWER>
inline cudaError_t trsm_sweep_nr(BatchT<C2> b, const C2* inv, C2* X, C2* Y, int nsys, int csize, cudaStream_t st,
                                 const int* active) {
  const int n = b.n, nblk = (n + TB - 1) / TB;
  constexpr int smem = sweep_smem<C2, NR>();
  static std::atomic<unsigned long long> attr{0};
  once_per_device(attr, [] {
    cudaFuncSetAttribute(trsm_sweep_kernel<C2, NR, LOWER>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nsys * csize), 1, 1);
  cfg.blockDim = dim3(SW_THREADS, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)csize;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, trsm_sweep_kernel<C2, NR, LOWER>, b, inv, nblk, X, Y, (long long)n * NR, active);
}

// ---------------------------------------------------------------------------
// Dataflow triangular sweep, one launch per direction. The 64-row blocks of
// every system are work items numbered level by level (forward: level l is
// block l; backward: block nbs-1-l); the systems still active at a level are a
// prefix of the batch (orders decrease along it). A persistent grid claims the
// items in that order with one atomic counter. An item accumulates the
// products of its row block with every solved block on the other side of the
// diagonal (left-looking), waiting on each source block's ready flag (the
// row block's loads are issued before the wait), solves with the inverted
// diagonal block, stores its block of the solution and raises its own flag.
// An item waits only on items of lower levels, which carry smaller numbers
// and were claimed by running CTAs before it, so the sweep always progresses
// whatever the number of resident CTAs. Every wait is bounded: one that runs
// out records ST_SWEEP_TIMEOUT in the status word and sets the abort word,
// which ends every other wait, so the launch always returns.
// Thread (r, g): row r of the block, column quarter g of each source block;
// the quarters' partial sums meet in shared memory.
// Workspace per direction: [0] item counter, [1] abort word,
// [2 + sys * nblk + blk] ready flags; zeroed before the launch.
// ---------------------------------------------------------------------------
constexpr int FL_THREADS = 256;
constexpr int FL_QUARTER = TB / 4;
constexpr int ST_SWEEP_TIMEOUT = 31;
constexpr long long FL_SPIN_LIMIT = 1LL << 21;

inline size_t flow_ws_ints(int nsys, int nblk) { return 2 + (size_t)nsys * nblk; }

// source blocks staged per wait (their solved blocks are loaded together)
constexpr int FL_CHUNK = 4;

template <class C2, int NR>
constexpr int flow_smem() {   // staged source blocks (later the quarters' partial sums), rhs block, inverse block
  return (FL_CHUNK * TB * NR + TB * NR + TB * TB) * (int)sizeof(C2);
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bounded wait for a ready flag (thread 0 of the CTA)
__device__ __forceinline__ void flow_wait(const int* flag, int* abort_w, int* status) {
  long long it = 0;
  while (ld_acquire(flag) == 0) {
    if (ld_acquire(abort_w)) return;
    if (++it > FL_SPIN_LIMIT) {
      if (status) atomicCAS(status, 0, ST_SWEEP_TIMEOUT);
      atomicExch(abort_w, 1);
      return;
    }
    __nanosleep(64);
  }
}

template <class C2, int NR, bool LOWER>
__global__ void __launch_bounds__(FL_THREADS) trsm_flow_kernel(BatchT<C2> b, const C2* __restrict__ inv, int nblk,
                                                               int nsys, const C2* __restrict__ R, C2* Y,
                                                               long long xstride, int* ws, int* status,
                                                               const int* active) {
  static_assert(FL_CHUNK >= 4, "the staging buffer also holds the four quarters' partial sums");
  if (active && *active == 0) return;   // a converged refinement skips its remaining passes
  extern __shared__ __align__(16) unsigned char fl_sm[];
  C2* yb = reinterpret_cast<C2*>(fl_sm);             // [FL_CHUNK][NR][TB] staged source blocks
  C2* red = yb;                                       // [4][NR][TB] partial sums, after the sources
  C2* rb = yb + FL_CHUNK * TB * NR;                   // [NR][TB] right-hand sides of the item's block
  C2* Ts = rb + TB * NR;                              // [TB][TB] inverse of its diagonal block
  int* pre = reinterpret_cast<int*>(Ts + TB * TB);    // [nblk + 1] items before each level
  __shared__ int s_item, s_nq;
  const int t = threadIdx.x, r = t % TB, g = t / TB;
  // systems active at level l: those with more than l blocks, a prefix
  for (int l = t; l < nblk; l += FL_THREADS) {
    int cnt = nsys;
    if (b.ord) {   // first system with at most l blocks (orders decrease along the batch)
      int lo = 0, hi = nsys;
      while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if ((b.ord[mid] + TB - 1) / TB > l) lo = mid + 1;
        else hi = mid;
      }
      cnt = lo;
    } else if (l >= (b.n + TB - 1) / TB) {
      cnt = 0;
    }
    pre[l + 1] = cnt;
  }
  __syncthreads();
  if (t == 0) {
    pre[0] = 0;
    for (int l = 0; l < nblk; ++l) pre[l + 1] += pre[l];
  }
  __syncthreads();
  const int total = pre[nblk];
  int* flags = ws + 2;
  for (;;) {
    // every thread has read the previous item before thread 0 claims the next
    // (an item of a converged system is skipped straight back to here)
    __syncthreads();
    if (t == 0) s_item = atomicAdd(ws, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= total) break;
    int lo = 0, hi = nblk;   // level: the last l with pre[l] <= item
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (pre[mid] <= item) lo = mid;
      else hi = mid;
    }
    const int sys = item - pre[lo];
    if (active && active[1 + sys] == 0) continue;   // a converged system: none of its items runs
    const int n = b.order(sys), nbs = (n + TB - 1) / TB;
    const int blk = LOWER ? lo : nbs - 1 - lo;
    const int k0 = blk * TB, nb = min(TB, n - k0);
    const C2* A = b.sys(sys);
    const C2* Rs = R + sys * xstride;
    C2* Ys = Y + sys * xstride;
    int* fl = flags + (long long)sys * nblk;
    // the item's right-hand sides and inverse block arrive while the sources are applied
    const C2* Ti = inv + ((long long)sys * nblk + blk) * 2 * TB * TB + (LOWER ? 0 : TB * TB);
    for (int e = t; e < TB * NR; e += FL_THREADS) {
      const int i = e % TB, p = e / TB;
      cp_async_elem(rb + e, i < nb ? Rs + (k0 + i) + (long long)n * p : Rs, i < nb);
    }
    for (int e = t; e < TB * TB; e += FL_THREADS) cp_async_elem(Ts + e, Ti + e, true);
    asm volatile("cp.async.commit_group;" ::: "memory");
    C2 acc[NR];
#pragma unroll
    for (int p = 0; p < NR; ++p) acc[p] = mkc<C2>(0., 0.);
    const int nsrc = LOWER ? blk : nbs - 1 - blk;
    auto src = [&](int q) { return LOWER ? q : nbs - 1 - q; };   // sources in the order they are solved
    auto load_row = [&](int q, C2* a) {   // this thread's 16 entries of the row block against source q
      const int c0 = src(q) * TB + g * FL_QUARTER;
#pragma unroll
      for (int j = 0; j < FL_QUARTER; ++j)
        a[j] = (r < nb && c0 + j < n) ? A[(k0 + r) + (long long)n * (c0 + j)] : mkc<C2>(0., 0.);
    };
    C2 an[FL_QUARTER];
    if (nsrc > 0) load_row(0, an);
#pragma unroll 1
    for (int q0 = 0, nq = 0; q0 < nsrc; q0 += nq) {
      // a chunk: the next source (waited for), then the sources after it
      // that are already solved, up to FL_CHUNK; the source an item waits on
      // last is thus applied as soon as it is ready, with nothing held back
      if (t == 0) {
        flow_wait(fl + src(q0), ws + 1, status);
        int m = 1;
        while (m < FL_CHUNK && q0 + m < nsrc && ld_acquire(fl + src(q0 + m))) ++m;
        s_nq = m;
      }
      __syncthreads();   // the flags are seen, and every thread is done with the previous chunk
      nq = s_nq;
      for (int e = t; e < nq * TB * NR; e += FL_THREADS) {
        const int qq = e / (TB * NR), m = e % (TB * NR), i = m % TB, p = m / TB;
        const int row = src(q0 + qq) * TB + i;
        yb[e] = row < n ? __ldcg(Ys + row + (long long)n * p) : mkc<C2>(0., 0.);
      }
      __syncthreads();
#pragma unroll 1
      for (int qq = 0; qq < nq; ++qq) {
        C2 a[FL_QUARTER];
#pragma unroll
        for (int j = 0; j < FL_QUARTER; ++j) a[j] = an[j];
        if (q0 + qq + 1 < nsrc) load_row(q0 + qq + 1, an);   // the next source's entries in flight
        const C2* y = yb + qq * TB * NR + g * FL_QUARTER;
#pragma unroll
        for (int j = 0; j < FL_QUARTER; ++j)
#pragma unroll
          for (int p = 0; p < NR; ++p) cmac(acc[p], a[j], y[j + TB * p]);
      }
    }
    __syncthreads();   // the staged sources are no longer read: the buffer takes the partial sums
#pragma unroll
    for (int p = 0; p < NR; ++p) red[(g * NR + p) * TB + r] = acc[p];
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    for (int e = t; e < TB * NR; e += FL_THREADS) {
      const int i = e % TB, p = e / TB;
      C2 v = rb[e];
#pragma unroll
      for (int gg = 0; gg < 4; ++gg) {
        const C2 u = red[(gg * NR + p) * TB + i];
        v.x -= u.x;
        v.y -= u.y;
      }
      rb[e] = i < nb ? v : mkc<C2>(0., 0.);
    }
    __syncthreads();
    // y = inv(T_blk) rb, the inverse's columns split by quarters like the sources
#pragma unroll
    for (int p = 0; p < NR; ++p) acc[p] = mkc<C2>(0., 0.);
#pragma unroll
    for (int j = 0; j < FL_QUARTER; ++j) {
      const int c = g * FL_QUARTER + j;
      const C2 ti = Ts[r + TB * c];
#pragma unroll
      for (int p = 0; p < NR; ++p) cmac(acc[p], ti, rb[c + TB * p]);
    }
    __syncthreads();   // every thread has read the partial sums it needed
#pragma unroll
    for (int p = 0; p < NR; ++p) red[(g * NR + p) * TB + r] = acc[p];
    __syncthreads();
    for (int e = t; e < TB * NR; e += FL_THREADS) {
      const int i = e % TB, p = e / TB;
      if (i < nb) {
        C2 v = red[p * TB + i];
#pragma unroll
        for (int gg = 1; gg < 4; ++gg) {
          const C2 u = red[(gg * NR + p) * TB + i];
          v.x += u.x;
          v.y += u.y;
        }
        Ys[(k0 + i) + (long long)n * p] = v;
      }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) st_release(fl + blk, 1);
  }
}

template <class C2, int NR, bool LOWER>
inline cudaError_t trsm_flow_nr(BatchT<C2> b, const C2* inv, const C2* R, C2* Y, int nsys, int* ws, int* status,
                                cudaStream_t st, const int* active) {
  const int nblk = (b.n + TB - 1) / TB;
  const int smem = flow_smem<C2, NR>() + (nblk + 1) * (int)sizeof(int);
  if (smem > 220 * 1024) return cudaErrorInvalidValue;
  auto kern = trsm_flow_kernel<C2, NR, LOWER>;
  static std::atomic<unsigned long long> attr{0};
  once_per_device(attr, [kern] { cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024); });
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // resident CTAs per SM for this shared-memory size (one query per size and device)
  static std::mutex mu;
  static std::map<long long, int> occ;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    const long long key = ((long long)dev << 32) | smem;
    auto it = occ.find(key);
    if (it != occ.end()) {
      per_sm = it->second;
    } else {
      cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FL_THREADS, smem);
      if (e != cudaSuccess) return e;
      occ[key] = per_sm;
    }
  }
  const long long items = (long long)nsys * nblk;
  const int grid = (int)std::max(1LL, std::min(items, (long long)std::max(1, sms) * std::max(1, per_sm)));
  kern<<<grid, FL_THREADS, smem, st>>>(b, inv, nblk, nsys, R, Y, (long long)b.n * NR, ws, status, active);
  return cudaGetLastError();
}

// the workspace both directions of one dataflow sweep use
struct SweepSync {
  int* ws = nullptr;       // 2 * flow_ws_ints(nsys, nblk) ints, or null: cluster sweep only
  int* status = nullptr;
};
constexpr int SWEEP_FLOW = 16;   // "cluster size" of the dataflow sweep in the tuner's choices

// Forward then backward sweep of nsys factored systems (nrhs right-hand sides
// in X, solution back in X, Y scratch of the same size): two launches.
// csize: the cluster sweep's cluster size (1..8), SWEEP_FLOW for the dataflow
// sweep (needs sync.ws), <= 0 for the default: the dataflow sweep when a
// workspace is given, else a cluster size from the device's SM count.
template <class C2>
inline cudaError_t trsm_sweep(BatchT<C2> b, const C2* inv, C2* X, C2* Y, int nsys, int nrhs, cudaStream_t st,
                              long long& launches, const int* active = nullptr, int csize = 0,
                              SweepSync sync = SweepSync()) {
  if (csize <= 0 && sync.ws) csize = SWEEP_FLOW;
  if (csize == SWEEP_FLOW && !sync.ws) csize = 0;
  if (csize <= 0) {
    static int sms = 0;
    if (!sms) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (sms <= 0) sms = 148;
    }
    csize = sweep_cluster(nsys, (b.n + TB - 1) / TB, sms);
  }
  cudaError_t e = cudaErrorInvalidValue;
  if (csize == SWEEP_FLOW) {
    const size_t wsn = flow_ws_ints(nsys, (b.n + TB - 1) / TB);
    e = cudaMemsetAsync(sync.ws, 0, 2 * wsn * sizeof(int), st);
    if (e != cudaSuccess) return e;
    switch (nrhs) {
#define NB200_FL(k)                                                                                     \
  case k:                                                                                               \
    e = trsm_flow_nr<C2, k, true>(b, inv, X, Y, nsys, sync.ws, sync.status, st, active);                \
    if (e == cudaSuccess) e = trsm_flow_nr<C2, k, false>(b, inv, Y, X, nsys, sync.ws + wsn, sync.status, st, active); \
    break;
      NB200_FL(1) NB200_FL(2) NB200_FL(3) NB200_FL(4) NB200_FL(5) NB200_FL(6) NB200_FL(7) NB200_FL(8)
      NB200_FL(9) NB200_FL(10) NB200_FL(11) NB200_FL(12) NB200_FL(13) NB200_FL(14) NB200_FL(15) NB200_FL(16)
#undef NB200_FL
      default:
        break;
    }
    launches += 2;
    return e;
  }
  switch (nrhs) {
#define NB200_SW(k)                                                                          \
  case k:                                                                                    \
    e = trsm_sweep_nr<C2, k, true>(b, inv, X, Y, nsys, csize, st, active);                   \
    if (e == cudaSuccess) e = trsm_sweep_nr<C2, k, false>(b, inv, Y, X, nsys, csize, st, active); \
    break;
    NB200_SW(1) NB200_SW(2) NB200_SW(3) NB200_SW(4) NB200_SW(5) NB200_SW(6) NB200_SW(7) NB200_SW(8)
    NB200_SW(9) NB200_SW(10) NB200_SW(11) NB200_SW(12) NB200_SW(13) NB200_SW(14) NB200_SW(15) NB200_SW(16)
#undef NB200_SW
    default:
      break;
  }
  launches += 2;
  return e;
}

// Y += sign * M X (FP64) with the columns split over blockIdx.y; partial sums
// are added with atomics, so Y must hold its initial value (0 or the RHS).
// The number of right-hand sides is a template parameter so that no
// predicated-off FMAs are issued (the kernel is balanced between HBM and the
// FP64 pipe at nine right-hand sides). Four CTAs per SM (128 registers, 16
// bytes of spills at nine right-hand sides instead of 132 registers and three
// CTAs) keep a third more column loads in flight: 9% less time per launch.
constexpr int MV_COLS = 128;
template <int NR>
__global__ void __launch_bounds__(128, 4) matvec_acc_kernel(Batch m, const double2* __restrict__ xbase, long long xstride,
                                                         double2* ybase, long long ystride, double sign,
                                                         const int* active) {
  if (active && *active == 0) return;   // a converged refinement skips its remaining passes
  if (active && active[1 + blockIdx.z] == 0) return;   // and a converged system its own work
  __shared__ double2 Xs[MV_COLS * NR];
  const int n = m.order(blockIdx.z);
  const double2* M = m.sys(blockIdx.z);
  const double2* X = xbase + blockIdx.z * xstride;
  const int c0 = blockIdx.y * MV_COLS, nc = min(MV_COLS, n - c0);
  if (nc <= 0 || (int)(blockIdx.x * blockDim.x) >= n) return;
  for (int q = threadIdx.x; q < MV_COLS * NR; q += blockDim.x) {
    const int c = q % MV_COLS, p = q / MV_COLS;
    Xs[c * NR + p] = (c < nc) ? X[(c0 + c) + (long long)n * p] : make_double2(0., 0.);
  }
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double2 acc[NR];
#pragma unroll
  for (int p = 0; p < NR; ++p) acc[p] = make_double2(0., 0.);
  const double2* Mr = M + r + (long long)n * c0;
  // the next 8 columns are loaded while the current 8 are multiplied
  double2 a[8], an[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = (j < nc) ? __ldg(Mr + (long long)n * j) : make_double2(0., 0.);
#pragma unroll 1
  for (int c8 = 0; c8 < nc; c8 += 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      an[j] = (c8 + 8 + j < nc) ? __ldg(Mr + (long long)n * (c8 + 8 + j)) : make_double2(0., 0.);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int p = 0; p < NR; ++p) cmad(acc[p], a[j], Xs[(c8 + j) * NR + p]);
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = an[j];
  }
  double2* Y = ybase + blockIdx.z * ystride;
#pragma unroll
  for (int p = 0; p < NR; ++p) {
    atomicAdd(&Y[r + (long long)n * p].x, sign * acc[p].x);
    atomicAdd(&Y[r + (long long)n * p].y, sign * acc[p].y);
  }
}

template <int NR>
inline void matvec_acc_nr(Batch m, const double2* x, long long xs, double2* y, long long ys, int nsys, double sign,
                          cudaStream_t st, const int* active) {
  const int n = m.n;
  matvec_acc_kernel<NR><<<dim3((n + 127) / 128, (n + MV_COLS - 1) / MV_COLS, nsys), 128, 0, st>>>(m, x, xs, y, ys,
                                                                                                  sign, active);
}

// Y += sign * M X for nsys systems with nrhs (1..MAX_RHS) right-hand sides;
// with `active` (refinement flags: [0] the launch, [1 + s] system s), nothing
// is done for a flag that is 0 on the device
inline void matvec_acc(Batch m, const double2* x, long long xs, double2* y, long long ys, int nrhs, int nsys,
                       double sign, cudaStream_t st, const int* active = nullptr) {
  switch (nrhs) {
#define NB200_MV(k)                                            \
  case k:                                                      \
    matvec_acc_nr<k>(m, x, xs, y, ys, nsys, sign, st, active); \
    break;
    NB200_MV(1) NB200_MV(2) NB200_MV(3) NB200_MV(4) NB200_MV(5) NB200_MV(6) NB200_MV(7) NB200_MV(8)
    NB200_MV(9) NB200_MV(10) NB200_MV(11) NB200_MV(12) NB200_MV(13) NB200_MV(14) NB200_MV(15) NB200_MV(16)
#undef NB200_MV
    default:
      break;
  }
}

}  // namespace nb200
