// Shared device/host definitions for the nemoh_b200 CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>

namespace nb200 {

// cudaFuncSetAttribute acts on the current device only, so a kernel that needs
// more dynamic shared memory than the default is set up once on every device
// a process uses; `done` holds one bit per device (concurrent first calls on a
// device may both set it, which is harmless).
// Grows a device allocation to at least n bytes. With headroom a quarter more
// is taken (n exactly if that does not fit): batches whose footprint keeps
// setting new maxima (cross-body batches of a request stream) then reallocate
// a few times instead of at every new maximum, each time a device-wide
// synchronisation (cudaFree) and a multi-GB cudaMalloc.
inline cudaError_t grow_alloc(void** p, size_t* have, size_t n, bool headroom) {
  if (n <= *have) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  size_t want = headroom ? n + n / 4 : n;
  cudaError_t e = cudaMalloc(p, want);
  if (e != cudaSuccess && want != n) {
    cudaGetLastError();
    want = n;
    e = cudaMalloc(p, want);
  }
  if (e == cudaSuccess) {
    *have = want;
  } else {
    *p = nullptr;
    // the failure goes back as the return value; consume it, so that a later
    // cudaGetLastError (a launch check) does not report it again
    cudaGetLastError();
  }
  return e;
}

template <class F>
inline void once_per_device(std::atomic<unsigned long long>& done, F set) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  set();
  done.fetch_or(bit, std::memory_order_acq_rel);
}


// ---------------------------------------------------------------------------
// Exactly rounded arithmetic for every quantity that decides a branch.
//
// The reference's Green functions switch formulas at thresholds (near/far
// field at RO = 7*TDIS, table stencil indices, AKZ/AKR ranges, ...). A one-ulp
// difference at a threshold flips a branch whose two sides differ by up to
// ~1e-2, so these quantities are computed with IEEE round-to-nearest
// intrinsics (no FMA contraction) in the same order as the FP64 oracle
// compiled with -ffp-contract=off. Values that only feed arithmetic use the
// fast path (FMA, CUDA libm).
// ---------------------------------------------------------------------------
#ifdef __CUDA_ARCH__
#define XADD(a, b) __dadd_rn((a), (b))
#define XSUB(a, b) __dsub_rn((a), (b))
#define XMUL(a, b) __dmul_rn((a), (b))
#define XDIV(a, b) __ddiv_rn((a), (b))
#define XSQRT(a) __dsqrt_rn((a))
#define NB_LDG(p) __ldg(p)
#else
// Host compilation of the same functions (the CPU check of the pair
// functions): IEEE double operations, built with -ffp-contract=off so that
// nothing is contracted into an FMA.
#define XADD(a, b) ((a) + (b))
#define XSUB(a, b) ((a) - (b))
#define XMUL(a, b) ((a) * (b))
#define XDIV(a, b) ((a) / (b))
#define XSQRT(a) std::sqrt((a))
#define NB_LDG(p) (*(p))
#endif
// functions of the Green-function family, compiled for the device and, for the
// CPU check, for the host
#define NB_HD __host__ __device__

struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, double s) { return {a.re + s, a.im}; }
__host__ __device__ __forceinline__ cplx operator+(double s, cplx a) { return {a.re + s, a.im}; }
__host__ __device__ __forceinline__ cplx operator-(double s, cplx a) { return {s - a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, double s) { return {a.re - s, a.im}; }
// Smith's algorithm (range-reduced division, as Fortran complex division)
__host__ __device__ __forceinline__ cplx operator/(cplx a, cplx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  double r = b.re / b.im, d = b.im + b.re * r;
  return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
__host__ __device__ __forceinline__ cplx operator/(double s, cplx b) { return mk(s, 0.0) / b; }
__host__ __device__ __forceinline__ cplx operator/(cplx a, double s) { return {a.re / s, a.im / s}; }
NB_HD __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
NB_HD __forceinline__ cplx cexp_(cplx a) {
  double e = exp(a.re), s, c;
  sincos(a.im, &s, &c);
  return {e * c, e * s};
}
NB_HD __forceinline__ cplx clog_(cplx a) { return {log(hypot(a.re, a.im)), atan2(a.im, a.re)}; }

// ---------------------------------------------------------------------------
// Table geometry (Solver/NEMOH.f90:179-208): 328 radial x 46 vertical nodes.
// ---------------------------------------------------------------------------
constexpr int TAB_IR = 328;
constexpr int TAB_JZ = 46;
constexpr int NPINTE = 251;
constexpr int MAX_NEXP = 31;
constexpr int MAX_NQ = 101;

// Stencil thresholds: integer stencil index = number of thresholds <= x.
// Computed on the host from the same log10 expressions the reference uses, so
// that the device reproduces the reference's truncation exactly.
struct StencilThresholds {
  double kj8[48];   // KJ=INT(8*(LOG10(x)+4.5)) >= k  <=>  x >= kj8[k]   (x=-AKZ > 1e-2)
  double kj5[48];   // KJ=INT(5*(LOG10(x)+6))   >= k  <=>  x >= kj5[k]   (x=-AKZ <= 1e-2)
  double ki5[48];   // KI=INT(5*(LOG10(y)+6)+1) >= k  <=>  y >= ki5[k]   (y=AKR+1e-20, AKR<1)
};

// Everything the kernels need about one frequency. Filled on the host.
struct OmegaParams {
  double w;        // W = 2*PI/T with T = 2*PI/omega (SOLVE_BEM.f90:62-63)
  double k0;       // infinite depth AK0 = W^2/G; finite depth AM0 = AMH/Depth
  double amh;      // finite depth m0*h
  double h;        // depth
  double coe1, coe2, coe3, coe4;  // VNSFD scale factors (COMPUTE_GREEN_FD.f90:259-268)
  int fd;          // 1 = finite depth path
  int nexp;        // number of fitted exponentials (finite depth)
  int nq;          // free-surface-panel theta quadrature length actually summed
  int pad;
  double ambda[MAX_NEXP + 1];  // 1-based like the reference; [nexp+1] = 0
  double ar[MAX_NEXP + 1];     // [nexp+1] = 2
  double cq[MAX_NQ + 1];       // theta weights (1-based)
  double ct[MAX_NQ + 1];       // cos(QQ) (1-based), computed on the host
  double st[MAX_NQ + 1];       // sin(QQ)
};

// Panel record staged per source panel J (PREPARE_MESH.f90 outputs + vertices)
struct PanelRec {
  double xg, yg, zg, xn, yn, zn, aire, tdis;
  double vx[4], vy[4], vz[4];
};

// Status codes (mirror include/nemoh_b200.h)
enum : int {
  ST_OK = 0, ST_INVALID = 1, ST_PANEL_AREA = 2, ST_PIVOT = 3, ST_OMEGA = 4, ST_LISC = 5, ST_SPRBM = 6,
  ST_DISPERSION = 7, ST_AKZ_UNDEFINED = 8, ST_IO = 9, ST_HOUSRS = 10, ST_CUDA = 20, ST_OOM = 21,
  ST_NO_DEVICE = 22, ST_CAPACITY = 23
};

}  // namespace nb200
