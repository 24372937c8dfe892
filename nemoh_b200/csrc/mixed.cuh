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
#include <map>
#include <vector>

#include "linalg.cuh"
#include "tc_gemm.cuh"
#include "tune.cuh"

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

// Refinement state on the device: decided by the last CTA of each residual
// pass, read by every later kernel of the refinement (which do nothing once
// `active` is 0) and by the host once per batch.
struct RefineState {
  int active;          // 1 while another pass is wanted
  int iterations;      // passes whose residual was measured
  int done_ctas;       // CTAs of the current residual pass that have finished
  int max_it;
  double worst;        // largest |r|inf / |b|inf of the last pass
  double prev;         // the same, one pass earlier
};

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
  RefineState* state = nullptr;         // refinement decisions on the device
  int* flow = nullptr;       // workspace of the dataflow sweep (both directions)
  int* act = nullptr;        // refinement activity: [0] another pass wanted, [1 + s] system s not converged yet
  int* status = nullptr;     // the owner's status word (sweep timeouts)
  TcWork tc;                 // tensor-core GEMM operand buffers
  size_t have[12] = {};      // bytes held by lu, diag, b, r, rf, yf, norms, inv, pinv, state, flow, act
  size_t total = 0;
  int last_iterations = 0;
  double last_residual = 0.;
  long long fallbacks = 0;   // batches re-solved with FP64 factors

  size_t bytes() const { return total; }
  void release() {
    cudaFree(lu); cudaFree(diag); cudaFree(b); cudaFree(r); cudaFree(rf); cudaFree(yf); cudaFree(norms); cudaFree(inv);
    cudaFree(pinv); cudaFree(state); cudaFree(flow); cudaFree(act);
    tc.release();
    lu = nullptr; diag = nullptr; b = nullptr; r = nullptr; rf = nullptr; yf = nullptr; norms = nullptr; inv = nullptr;
    pinv = nullptr; state = nullptr; flow = nullptr; act = nullptr;
    for (size_t& h : have) h = 0;
    total = 0;
  }
  ~MixedWork() { release(); }
  // Each buffer grows on its own when the batch needs more bytes than it holds
  // (strides always follow the current n), so a smaller mesh with more
  // systems reuses what a larger one left and nothing is freed needlessly:
  // cudaFree synchronizes the whole device.
  // mat_elems: elements of all matrices of a ragged batch (0: nsys x n x n)
  // headroom: see grow_alloc (cross-body batches)
  cudaError_t ensure(int nsys, int n, int nrhs, size_t mat_elems = 0, bool headroom = false) {
    const size_t NN = (size_t)n * n, V = (size_t)nsys * n * nrhs;
    const size_t need[12] = {(mat_elems ? mat_elems : nsys * NN) * sizeof(float2),
                            (size_t)nsys * DIAG_SCRATCH * sizeof(float2),
                            V * sizeof(double2),
                            V * sizeof(double2),
                            V * sizeof(float2),
                            V * sizeof(float2),
                            (size_t)2 * nsys * nrhs * sizeof(unsigned long long),
                            (size_t)nsys * ((n + TB - 1) / TB) * 2 * TB * TB * sizeof(float2),
                            (size_t)nsys * PINV_SCRATCH * sizeof(float2),
                            sizeof(RefineState),
                            2 * flow_ws_ints(nsys, (n + TB - 1) / TB) * sizeof(int),
                            (size_t)(1 + nsys) * sizeof(int)};
    void** ptr[12] = {(void**)&lu, (void**)&diag, (void**)&b, (void**)&r, (void**)&rf, (void**)&yf, (void**)&norms,
                      (void**)&inv, (void**)&pinv, (void**)&state, (void**)&flow, (void**)&act};
    for (int i = 0; i < 12; ++i) {
      cudaError_t e = grow_alloc(ptr[i], &have[i], need[i], headroom);
      if (e) return e;
    }
    cudaError_t e = tc.ensure(nsys, n, headroom);
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

// |b|inf per (system, rhs). Vectors of system s start at s * nrhs * n (n =
// the largest order of a ragged batch, `ord` its systems' orders, or null)
// with leading dimension the system's own order.
__global__ void norm_kernel(const double2* __restrict__ v, int n, int nrhs, unsigned long long* out,
                            const int* __restrict__ ord) {
  const int p = blockIdx.y, s = blockIdx.z;
  const double2* x = v + (long long)s * nrhs * n + (long long)p * (ord ? ord[s] : n);
  if (ord) n = ord[s];
  double m = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y)));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out + (long long)s * nrhs + p, (unsigned long long)__double_as_longlong(m));
}

// the block panel's products L21 = A21 inv(U11) and U12 = inv(L11) A12 on the
// tensor cores (NEMOH_B200_TC_PRODUCTS=0: on the CUDA cores)
inline bool tc_products_on() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_TC_PRODUCTS");
    return !(e && e[0] == '0');
  }();
  return on;
}

// merged outer updates of panel pairs (NEMOH_B200_TC_MERGE=0 turns them off)
inline bool tc_merge() {
  static const bool on = [] {
    const char* e = std::getenv("NEMOH_B200_TC_MERGE");
    return !(e && e[0] == '0');
  }();
  return on;
}

// have_f32: the assembly already wrote the FP32 copy of D into w.lu
// rg: ragged batch (systems sorted by decreasing order, n the largest; the
// FP32 copy in w.lu has the same element offsets as D); mat_elems: elements
// of all matrices (for the conversion when the copy is not there yet)
// sys0 (uniform batches): factor systems [sys0, sys0 + nsys) of the batch, in
// their own slices of every per-system buffer, so that two ranges of one
// batch can be factored on two streams at once
inline void mixed_factor(MixedWork& w, double2* D, int n, int nsys, int* status, cudaStream_t st, long long& launches,
                         const Lanes* lanes = nullptr, bool have_f32 = false, const Ragged& rg = Ragged(),
                         long long mat_elems = -1, int sys0 = 0) {
  const size_t NN = (size_t)n * n, tiles = (size_t)(n + TC_T - 1) / TC_T;
  const int nblk = (n + TB - 1) / TB;
  float2* lu = w.lu + sys0 * NN;
  if (!have_f32) {
    const long long total = mat_elems >= 0 ? mat_elems : (long long)nsys * n * n;
    d2f_kernel<<<1184, 256, 0, st>>>(D + sys0 * NN, lu, total);
    ++launches;
  }
  BatchT<float2> b = make_batch<float2>(lu, n, w.diag + (size_t)sys0 * DIAG_SCRATCH,
                                        w.pinv + (size_t)sys0 * PINV_SCRATCH, rg);
  float2* inv = w.inv + (size_t)sys0 * nblk * 2 * TB * TB;
  // Merged outer updates (persistent tensor-core form): after an even panel
  // whose next panel still has columns beyond it, only the next panel's
  // columns (all rows) and the next panel's rows (the columns beyond) are
  // updated; the rest of the trailing matrix takes both panels' products in
  // the next panel's update (K = 256), so each pair of panels reads and
  // writes the bulk of A22 once. deferred: per group (by its first system),
  // the image set holding the deferred panel's images, or -1.
  const bool merge = tc_enabled() && tc_persistent() && tc_merge();
  // the block path's L21 and U12 products on the tensor cores too
  const bool tc_prod = tc_enabled() && tc_persistent() && tc_products_on() && panel_as_block() && w.pinv;
  std::map<int, int> deferred;
  lu_two_level<float2>(
      b, nsys, status, st, launches,
      [&](BatchT<float2> bg, int ns, cudaStream_t sg, int s0, int k0, int kend) {
        // the group's slice of each image set
        auto slice = [&](int set) {
          TcWork tg = w.tc.set(set);
          tg.a += (size_t)(sys0 + s0) * tiles * TC_NCH * 2 * TC_AIMG;
          tg.b += (size_t)(sys0 + s0) * tiles * TC_NCH * 2 * TC_BIMG;
          tg.wv += (size_t)(sys0 + s0) * TC_WV_BYTES;
          return tg;
        };
        if (!tc_enabled()) {
          zgemm_update<float2>(bg, k0, kend - k0, Rect{kend, bg.n, kend, bg.n}, ns, sg);
          ++launches;
          return;
        }
        const int set = (k0 / LU_OUTER) & 1;
        TcWork tg = slice(set);
        // operand images of the panel's columns and rows: with tc_prod those of
        // A21 and A12, from which the block products form L21 = A21 V and
        // U12 = W A12 together with their images; else those of L21 and U12
        tc_prep(tg, bg, k0, ns, sg, launches);
        if (tc_prod) tc_products(tg, bg, k0, ns, sg, launches, status);
        if (!merge) {
          tc_apply(tg, bg, k0, ns, sg, launches, status, TcTiles(), tc_persistent());
          return;
        }
        auto it = deferred.find(s0);
        if (it != deferred.end() && it->second >= 0) {   // this panel's update and the deferred one
          const TcWork prev = slice(it->second);
          tc_apply(tg, bg, k0, ns, sg, launches, status, TcTiles(), true, &prev);
          it->second = -1;
        } else if (kend + LU_OUTER < bg.n) {   // the next panel has columns beyond it: defer the bulk
          tc_apply(tg, bg, k0, ns, sg, launches, status, TcTiles{0, -1, 0, 1}, true);
          tc_apply(tg, bg, k0, ns, sg, launches, status, TcTiles{0, 1, 1, -1}, true);
          deferred[s0] = set;
        } else {
          tc_apply(tg, bg, k0, ns, sg, launches, status, TcTiles(), true);
        }
      },
      lanes, rg.host_ord, tc_prod);
  static std::atomic<unsigned long long> attr{0};
  once_per_device(attr, [] {
    cudaFuncSetAttribute(inv_diag_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         inv_diag_smem<float2>());
  });
  inv_diag_kernel<float2><<<dim3(nblk, 1, nsys), INV_THREADS, inv_diag_smem<float2>(), st>>>(b, inv, nblk);
  ++launches;
}

inline void trsm_f32(MixedWork& w, int n, int nsys, int nrhs, cudaStream_t st, long long& launches,
                     const int* active, const Ragged& rg) {
  BatchT<float2> b = make_batch<float2>(w.lu, n, w.diag, nullptr, rg);
  trsm_sweep_tuned<float2>(b, w.inv, w.rf, w.yf, nsys, nrhs, st, launches, active, SweepSync{w.flow, w.status});
  // the solution is left in w.rf (forward into yf, backward back into rf)
}

__global__ void refine_start_kernel(RefineState* st, int max_it) {
  st->active = 1;
  st->iterations = 0;
  st->done_ctas = 0;
  st->max_it = max_it;
  st->worst = 1e300;
  st->prev = 1e300;
}

// x += correction (x = correction on the first pass), r = b, residual norms
// cleared for the coming residual pass; systems that have converged (act[1 +
// s] == 0, s = q / xs) keep their solution and leave their norms at 0
__global__ void refine_update_kernel(double2* __restrict__ x, const float2* __restrict__ d,
                                     const double2* __restrict__ b, double2* __restrict__ r, long long count,
                                     long long xs, unsigned long long* __restrict__ rnorm, int nv,
                                     const RefineState* st, const int* __restrict__ act) {
  if (!st->active) return;
  const int first = st->iterations == 0;
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
  for (long long q = t0; q < nv; q += stride) rnorm[q] = 0ull;
  for (long long q = t0; q < count; q += stride) {
    if (act[1 + q / xs] == 0) continue;
    const float2 v = d[q];
    if (first) x[q] = make_double2(v.x, v.y);
    else {
      double2 o = x[q];
      o.x += v.x;
      o.y += v.y;
      x[q] = o;
    }
    r[q] = b[q];
  }
}

// rf = (float) r and |r|inf per (system, rhs), r = b - D x formed beforehand;
// the last CTA to finish compares the largest relative residual with the
// tolerance and the previous pass (no CTA waits on another: the decision is
// taken by whichever CTA counts itself last, after a fence)
__global__ void __launch_bounds__(256) refine_residual_kernel(const double2* __restrict__ r, float2* __restrict__ rf,
                                                              int n, int nrhs, unsigned long long* __restrict__ norms,
                                                              int nv, RefineState* st, double tol,
                                                              const int* __restrict__ ord, int* act) {
  if (!st->active) return;
  const int p = blockIdx.y, s = blockIdx.z;
  const long long base = (long long)s * nrhs * n + (long long)p * (ord ? ord[s] : n);
  const bool mine = act[1 + s] != 0;   // a converged system's CTAs only count themselves
  if (ord) n = ord[s];
  double m = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; mine && i < n; i += gridDim.x * blockDim.x) {
    const double2 v = r[base + i];
    rf[base + i] = make_float2((float)v.x, (float)v.y);
    // a NaN component counts as infinite (fmax would drop it), so a failed
    // factorization can never pass for a converged one
    m = fmax(m, (v.x == v.x && v.y == v.y) ? fmax(fabs(v.x), fabs(v.y)) : HUGE_VAL);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(norms + (long long)s * nrhs + p, (unsigned long long)__double_as_longlong(m));
  __threadfence();
  __syncthreads();
  __shared__ int last;
  if (threadIdx.x == 0) {
    const int total = gridDim.x * gridDim.y * gridDim.z;
    last = atomicAdd(&st->done_ctas, 1) == total - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double worst = 0.;
  for (int q = threadIdx.x; q < nv; q += blockDim.x) {
    const double rn = __longlong_as_double((long long)atomicAdd(norms + q, 0ull));
    const double bn = __longlong_as_double((long long)norms[nv + q]);
    worst = fmax(worst, bn > 0 ? rn / bn : rn);
  }
  __shared__ double red[256];
  red[threadIdx.x] = worst;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  __shared__ int s_stop;
  if (threadIdx.x == 0) {
    const double w = red[0];
    const int it = st->iterations + 1;
    st->iterations = it;
    st->worst = w;
    // stop at the tolerance, or as soon as the residual no longer halves
    // (stagnation or divergence: the host then falls back to FP64 factors)
    const bool stop = w <= tol || !(w == w) || w > 0.5 * st->prev || it >= st->max_it;
    st->prev = w;
    st->done_ctas = 0;
    st->active = stop ? 0 : 1;
    act[0] = stop ? 0 : 1;
    s_stop = stop;
  }
  __syncthreads();
  // the next pass works only on the systems still above the tolerance
  const int nsys = gridDim.z;
  for (int sy = threadIdx.x; sy < nsys; sy += blockDim.x) {
    double ws = 0.;
    for (int q = sy * nrhs; q < (sy + 1) * nrhs; ++q) {
      const double rn = __longlong_as_double((long long)atomicAdd(norms + q, 0ull));
      const double bn = __longlong_as_double((long long)norms[nv + q]);
      ws = fmax(ws, bn > 0 ? rn / bn : rn);
    }
    act[1 + sy] = (!s_stop && !(ws <= tol)) ? 1 : 0;
  }
}

// Passes issued per host check: the refinement normally meets the tolerance in
// two or three, and a pass issued after convergence costs only its launches.
constexpr int REFINE_CHUNK = 4;

// The refinement in two halves so that a captured launch sequence can hold
// it: mixed_refine_begin issues the set-up, mixed_refine_passes issues passes
// without any host synchronisation (each pass's last residual kernel decides
// on the device whether another is wanted, and the passes after that decision
// do nothing), mixed_refine_read reads the decision.
struct RefineArgs {
  double2* D;      // FP64 matrices (the residual's operator)
  int n, nsys, nrhs;
  double2* X;      // right-hand sides in, solution out (FP64)
  Ragged rg;
};

inline void mixed_refine_begin(MixedWork& w, const RefineArgs& a, int max_it, cudaStream_t st, long long& launches) {
  const long long V = (long long)a.nsys * a.n * a.nrhs;
  const int nv = a.nsys * a.nrhs;
  cudaMemcpyAsync(w.b, a.X, V * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(w.norms, 0, 2 * (size_t)nv * sizeof(unsigned long long), st);
  norm_kernel<<<dim3(4, a.nrhs, a.nsys), 256, 0, st>>>(w.b, a.n, a.nrhs, w.norms + nv, a.rg.ord);
  ++launches;
  d2f_kernel<<<1184, 256, 0, st>>>(w.b, w.rf, V);
  ++launches;
  refine_start_kernel<<<1, 1, 0, st>>>(w.state, max_it);
  ++launches;
  cudaMemsetAsync(w.act, 1, (size_t)(1 + a.nsys) * sizeof(int), st);   // nonzero: every system active
}

inline void mixed_refine_passes(MixedWork& w, const RefineArgs& a, int passes, cudaStream_t st, long long& launches) {
  const long long V = (long long)a.nsys * a.n * a.nrhs, xs = (long long)a.n * a.nrhs;
  const int nv = a.nsys * a.nrhs;
  const Batch dm = make_batch<double2>(a.D, a.n, nullptr, nullptr, a.rg);
  // act: [0] another pass wanted, [1 + s] system s still above the tolerance
  const int* active = w.act;
  for (int it = 0; it < passes; ++it) {
    trsm_f32(w, a.n, a.nsys, a.nrhs, st, launches, active, a.rg);
    refine_update_kernel<<<1184, 256, 0, st>>>(a.X, w.rf, w.b, w.r, V, xs, w.norms, nv, w.state, w.act);
    ++launches;
    matvec_acc(dm, a.X, xs, w.r, xs, a.nrhs, a.nsys, -1.0, st, active);
    ++launches;
    refine_residual_kernel<<<dim3(8, a.nrhs, a.nsys), 256, 0, st>>>(w.r, w.rf, a.n, a.nrhs, w.norms, nv, w.state,
                                                                    REFINE_TOL, a.rg.ord, w.act);
    ++launches;
  }
}

// waits for the stream; returns true while the device still wants passes
inline bool mixed_refine_read(MixedWork& w, cudaStream_t st) {
  RefineState h{};
  cudaMemcpyAsync(&h, w.state, sizeof h, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  w.last_iterations = h.iterations;
  w.last_residual = h.worst;
  return h.active != 0;
}

// X: right-hand sides in, solution out (FP64). Passes are issued
// REFINE_CHUNK at a time, with one host check per chunk.
inline void mixed_solve_refine(MixedWork& w, double2* D, int n, int nsys, double2* X, double2* /*Y*/, int nrhs,
                               cudaStream_t st, long long& launches, const Ragged& rg = Ragged()) {
  const RefineArgs a{D, n, nsys, nrhs, X, rg};
  const int max_it = refine_max_it();
  mixed_refine_begin(w, a, max_it, st, launches);
  for (int it0 = 0; it0 < max_it; it0 += REFINE_CHUNK) {
    mixed_refine_passes(w, a, std::min(REFINE_CHUNK, max_it - it0), st, launches);
    if (!mixed_refine_read(w, st)) break;
  }
}

}  // namespace nb200
