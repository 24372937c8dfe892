// Mixed-precision solve: low-precision LU of the influence matrix, FP64
// iterative refinement against the FP64 matrix.
//
// x0 = LU32^-1 b;  repeat  r = b - D x (FP64 residual, FP64 matrix D),
//                          x += LU32^-1 r   until |r|inf <= tol |b|inf.
// The FP32 factorization is the blocked no-pivot LU of linalg.cuh in two
// levels: 128-column panels are factored with 32-column steps whose updates
// stay inside the panel and its row strip (FP32 SIMT), and the rest of the
// trailing matrix is updated once per panel with K = 128 on the tensor cores
// (tc_gemm.cuh: split-BF16 operands, FP32 accumulation), or as an FP32 SIMT
// GEMM when the tcgen05 path is disabled.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "linalg.cuh"
#include "tc_gemm.cuh"

namespace nb200 {

constexpr int REFINE_MAX_IT = 30;

// iteration limit: NEMOH_B200_REFINE_MAX_IT overrides the default (tests use a
// small limit to exercise the FP64 fallback)
inline int refine_max_it() {
  const char* e = std::getenv("NEMOH_B200_REFINE_MAX_IT");
  const int v = e ? std::atoi(e) : 0;
  return v > 0 ? v : REFINE_MAX_IT;
}
// A batch is accepted when its largest relative residual |b - D x|inf/|b|inf
// is at most REFINE_TOL. The error of x is at most cond(D) times that, below
// 1e-8 for the conditioning met on hull meshes away from irregular
// frequencies; near one the FP32 factors stall or diverge and the batch is
// solved again with FP64 factors.
constexpr double REFINE_TOL = 1e-12;

struct MixedWork {
  float2* lu = nullptr;      // FP32 factors, nsys x n x n
  float2* diag = nullptr;    // diagonal-block scratch (factors and inverses)
  double2* b = nullptr;      // right-hand sides (FP64)
  double2* r = nullptr;      // residual (FP64)
  float2* rf = nullptr;      // residual/correction (FP32)
  float2* yf = nullptr;      // forward-solve scratch (FP32)
  float2* inv = nullptr;     // inverses of the diagonal blocks of L and U (FP32)
  float2* pinv = nullptr;    // inv(L) of the diagonal blocks of the current outer panel
  unsigned long long* norms = nullptr;  // |r|inf bits per system and rhs, then |b|inf
  TcWork tc;                 // tensor-core GEMM operand buffers
  size_t have[9] = {};       // bytes held by lu, diag, b, r, rf, yf, norms, inv, pinv
  size_t total = 0;
  int last_iterations = 0;
  double last_residual = 0.;
  long long fallbacks = 0;   // batches re-solved with FP64 factors

  size_t bytes() const { return total; }
  void release() {
    cudaFree(lu); cudaFree(diag); cudaFree(b); cudaFree(r); cudaFree(rf); cudaFree(yf); cudaFree(norms); cudaFree(inv);
    cudaFree(pinv);
    tc.release();
    lu = nullptr; diag = nullptr; b = nullptr; r = nullptr; rf = nullptr; yf = nullptr; norms = nullptr; inv = nullptr;
    pinv = nullptr;
    for (size_t& h : have) h = 0;
    total = 0;
  }
  ~MixedWork() { release(); }
  // Each buffer grows on its own when the batch needs more bytes than it holds
  // (strides always follow the current n), so a smaller mesh with more
  // systems reuses what a larger one left and nothing is freed needlessly:
  // cudaFree synchronizes the whole device.
  cudaError_t ensure(int nsys, int n, int nrhs) {
    const size_t NN = (size_t)n * n, V = (size_t)nsys * n * nrhs;
    const size_t need[9] = {nsys * NN * sizeof(float2),
                            (size_t)nsys * DIAG_SCRATCH * sizeof(float2),
                            V * sizeof(double2),
                            V * sizeof(double2),
                            V * sizeof(float2),
                            V * sizeof(float2),
                            (size_t)2 * nsys * nrhs * sizeof(unsigned long long),
                            (size_t)nsys * ((n + TB - 1) / TB) * 2 * TB * TB * sizeof(float2),
                            (size_t)nsys * PINV_SCRATCH * sizeof(float2)};
    void** ptr[9] = {(void**)&lu, (void**)&diag, (void**)&b, (void**)&r, (void**)&rf, (void**)&yf, (void**)&norms,
                     (void**)&inv, (void**)&pinv};
    for (int i = 0; i < 9; ++i) {
      if (need[i] <= have[i]) continue;
      cudaFree(*ptr[i]);
      *ptr[i] = nullptr;
      have[i] = 0;
      cudaError_t e = cudaMalloc(ptr[i], need[i]);
      if (e) return e;
      have[i] = need[i];
    }
    cudaError_t e = tc.ensure(nsys, n);
    if (e) return e;
    total = tc.bytes();
    for (size_t h : have) total += h;
    return cudaSuccess;
  }
};

inline size_t mixed_bytes_per_system(size_t n) {
  return n * n * sizeof(float2) + tc_bytes_per_system(n) + ((n + TB - 1) / TB) * 2 * TB * TB * sizeof(float2) +
         (DIAG_SCRATCH + PINV_SCRATCH) * sizeof(float2);
}

__global__ void d2f_kernel(const double2* __restrict__ a, float2* __restrict__ b, long long count) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < count; q += (long long)gridDim.x * blockDim.x) {
    const double2 v = a[q];
    b[q] = make_float2((float)v.x, (float)v.y);
  }
}

// x += correction (FP32 -> FP64); on the first pass x = correction
__global__ void accumulate_kernel(double2* __restrict__ x, const float2* __restrict__ d, long long count, int first) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < count; q += (long long)gridDim.x * blockDim.x) {
    const float2 v = d[q];
    if (first) x[q] = make_double2(v.x, v.y);
    else {
      double2 o = x[q];
      o.x += v.x;
      o.y += v.y;
      x[q] = o;
    }
  }
}

// |b|inf per (system, rhs)
__global__ void norm_kernel(const double2* __restrict__ v, int n, int nrhs, unsigned long long* out) {
  const int p = blockIdx.y, s = blockIdx.z;
  const double2* x = v + ((long long)s * nrhs + p) * n;
  double m = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y)));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out + (long long)s * nrhs + p, (unsigned long long)__double_as_longlong(m));
}

// rf = (float) r and |r|inf per (system, rhs), r = b - D x formed beforehand
__global__ void residual_finish_kernel(const double2* __restrict__ r, float2* __restrict__ rf, int n, int nrhs,
                                       unsigned long long* __restrict__ rnorm) {
  const int p = blockIdx.y, s = blockIdx.z;
  const long long base = ((long long)s * nrhs + p) * n;
  double m = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 v = r[base + i];
    rf[base + i] = make_float2((float)v.x, (float)v.y);
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(rnorm + (long long)s * nrhs + p, (unsigned long long)__double_as_longlong(m));
}

// have_f32: the assembly already wrote the FP32 copy of D into w.lu
inline void mixed_factor(MixedWork& w, double2* D, int n, int nsys, int* status, cudaStream_t st, long long& launches,
                         const Lanes* lanes = nullptr, bool have_f32 = false) {
  if (!have_f32) {
    const long long total = (long long)nsys * n * n;
    d2f_kernel<<<1184, 256, 0, st>>>(D, w.lu, total);
    ++launches;
  }
  BatchT<float2> b{w.lu, (long long)n * n, n, w.diag, w.pinv};
  const size_t tiles = (size_t)(n + TC_T - 1) / TC_T;
  lu_two_level<float2>(
      b, nsys, status, st, launches,
      [&](BatchT<float2> bg, int ns, cudaStream_t sg, int s0, int k0, int kend) {
        TcWork tg = w.tc;   // the group's slice of the operand images
        tg.a += (size_t)s0 * tiles * TC_NCH * 2 * TC_AIMG;
        tg.b += (size_t)s0 * tiles * TC_NCH * 2 * TC_BIMG;
        if (!tc_update(tg, bg, k0, ns, sg, launches, status)) {
          zgemm_update<float2>(bg, k0, kend - k0, Rect{kend, n, kend, n}, ns, sg);
          ++launches;
        }
      },
      lanes);
  static std::atomic<unsigned long long> attr{0};
  once_per_device(attr, [] {
    cudaFuncSetAttribute(inv_diag_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         inv_diag_smem<float2>());
  });
  const int nblk = (n + TB - 1) / TB;
  inv_diag_kernel<float2><<<dim3(nblk, 1, nsys), INV_THREADS, inv_diag_smem<float2>(), st>>>(b, w.inv, nblk);
  ++launches;
}

inline void trsm_f32(MixedWork& w, int n, int nsys, int nrhs, cudaStream_t st, long long& launches,
                     const Lanes* lanes) {
  BatchT<float2> b{w.lu, (long long)n * n, n, w.diag};
  trsm_launch<float2>(b, w.inv, w.rf, w.yf, nsys, nrhs, st, launches, lanes);
  // the solution is left in w.rf (forward into yf, backward back into rf)
}

// X: right-hand sides in, solution out (FP64); Y unused scratch
inline void mixed_solve_refine(MixedWork& w, double2* D, int n, int nsys, double2* X, double2* /*Y*/, int nrhs,
                               cudaStream_t st, long long& launches, const Lanes* lanes = nullptr) {
  const long long V = (long long)nsys * n * nrhs;
  const int nv = nsys * nrhs;
  cudaMemcpyAsync(w.b, X, V * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(w.norms, 0, 2 * (size_t)nv * sizeof(unsigned long long), st);
  norm_kernel<<<dim3(4, nrhs, nsys), 256, 0, st>>>(w.b, n, nrhs, w.norms + nv);
  ++launches;
  d2f_kernel<<<1184, 256, 0, st>>>(w.b, w.rf, V);
  ++launches;
  std::vector<unsigned long long> h(2 * (size_t)nv);
  Batch dm{D, (long long)n * n, n, nullptr};
  w.last_iterations = 0;
  const int max_it = refine_max_it();
  double prev = 1e300;
  for (int it = 0; it < max_it; ++it) {
    trsm_f32(w, n, nsys, nrhs, st, launches, lanes);
    accumulate_kernel<<<1184, 256, 0, st>>>(X, w.rf, V, it == 0);
    ++launches;
    cudaMemsetAsync(w.norms, 0, (size_t)nv * sizeof(unsigned long long), st);
    cudaMemcpyAsync(w.r, w.b, V * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    matvec_acc(dm, X, (long long)n * nrhs, w.r, (long long)n * nrhs, nrhs, nsys, -1.0, st);
    ++launches;
    residual_finish_kernel<<<dim3(8, nrhs, nsys), 256, 0, st>>>(w.r, w.rf, n, nrhs, w.norms);
    ++launches;
    cudaMemcpyAsync(h.data(), w.norms, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    double worst = 0.;
    for (int q = 0; q < nv; ++q) {
      double rn, bn;
      std::memcpy(&rn, &h[q], 8);
      std::memcpy(&bn, &h[nv + q], 8);
      worst = std::max(worst, bn > 0 ? rn / bn : rn);
    }
    w.last_iterations = it + 1;
    w.last_residual = worst;
    // stop at the tolerance, or as soon as the residual no longer halves
    // (stagnation or divergence: the caller then falls back to FP64 factors)
    if (worst <= REFINE_TOL || !(worst == worst) || worst > 0.5 * prev) break;
    prev = worst;
  }
}

}  // namespace nb200
