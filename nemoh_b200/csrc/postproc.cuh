// Radiation impulse response functions of the post-processor
// (postProcessor/IRF.f90:100-127, Compute_IRF):
//   K(t_i) = 2/pi sum_l 0.5 (B_l cos(w_l t_i) + B_l+1 cos(w_l+1 t_i)) (w_l+1 - w_l)
//   A_inf  = 1/Nw sum_l [A_l + 1/w_l sum_i 0.5 (K_i sin(w_l t_i) + K_i+1 sin(w_l t_i+1)) dt]
// with t_i = i dt. Coefficients are (Nw, Nrad, Nint) with w fastest, K is
// (Ntime, Nrad, Nint) with time fastest. Each thread owns one time (or one
// frequency) and up to IRF_CH radiation/force pairs, so every cos/sin is
// evaluated once per pair chunk; each sum runs in the reference's order.
#pragma once
#include "common.cuh"

namespace nb200 {

constexpr int IRF_CH = 16;
constexpr int IRF_THREADS = 128;

// K: grid (ceil(ntime / 128), ceil(npair / IRF_CH))
__global__ void __launch_bounds__(IRF_THREADS)
    irf_kernel(int nw, const double* __restrict__ w, int npair, const double* __restrict__ damping, int ntime,
               double dt, double* __restrict__ K) {
  const int i = blockIdx.x * IRF_THREADS + threadIdx.x;
  const int p0 = blockIdx.y * IRF_CH, np = min(IRF_CH, npair - p0);
  if (i >= ntime) return;
  const double t = i * dt;
  double acc[IRF_CH];
#pragma unroll
  for (int q = 0; q < IRF_CH; ++q) acc[q] = 0.;
  double c0 = cos(w[0] * t);
  for (int l = 0; l < nw - 1; ++l) {
    const double c1 = cos(w[l + 1] * t), dw = w[l + 1] - w[l];
#pragma unroll
    for (int q = 0; q < IRF_CH; ++q) {
      if (q >= np) break;
      const double* B = damping + (size_t)nw * (p0 + q);
      acc[q] = acc[q] + 0.5 * (B[l] * c0 + B[l + 1] * c1) * dw;
    }
    c0 = c1;
  }
  const double PI = 4. * atan(1.0);
#pragma unroll
  for (int q = 0; q < IRF_CH; ++q) {
    if (q >= np) break;
    K[i + (size_t)ntime * (p0 + q)] = acc[q] * 2. / PI;
  }
}

// CM(l, pair) = A_l + (trapezoid of K sin(w_l t)) / w_l: grid (ceil(nw / 128), ceil(npair / IRF_CH))
__global__ void __launch_bounds__(IRF_THREADS)
    irf_added_mass_kernel(int nw, const double* __restrict__ w, int npair, const double* __restrict__ added_mass,
                          int ntime, double dt, const double* __restrict__ K, double* __restrict__ cm) {
  const int l = blockIdx.x * IRF_THREADS + threadIdx.x;
  const int p0 = blockIdx.y * IRF_CH, np = min(IRF_CH, npair - p0);
  if (l >= nw) return;
  const double wl = w[l];
  double acc[IRF_CH];
#pragma unroll
  for (int q = 0; q < IRF_CH; ++q) acc[q] = 0.;
  double s0 = sin(wl * 0.);
  for (int i = 0; i < ntime - 1; ++i) {
    const double t0 = i * dt, t1 = (i + 1) * dt;
    const double s1 = sin(wl * t1);
#pragma unroll
    for (int q = 0; q < IRF_CH; ++q) {
      if (q >= np) break;
      const double* Kp = K + (size_t)ntime * (p0 + q);
      acc[q] = acc[q] + 0.5 * (Kp[i] * s0 + Kp[i + 1] * s1) * (t1 - t0);
    }
    s0 = s1;
  }
#pragma unroll
  for (int q = 0; q < IRF_CH; ++q) {
    if (q >= np) break;
    cm[l + (size_t)nw * (p0 + q)] = added_mass[l + (size_t)nw * (p0 + q)] + acc[q] / wl;
  }
}

// A_inf(pair) = sum_l CM(l, pair) / nw, summed in frequency order
__global__ void irf_average_kernel(int nw, int npair, const double* __restrict__ cm, double* __restrict__ ainf) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npair) return;
  double am = 0.;
  for (int l = 0; l < nw; ++l) am = am + cm[l + (size_t)nw * p];
  ainf[p] = am / nw;
}

}  // namespace nb200
