// Kochin function of the solved problems (COMPUTE_KOCHIN.f90:25-152).
//
// H(theta) = 1/(4 pi) sum_J [ ZIGB(J) ZS_J(theta) + ZIGS(J) ZS'_J(theta) ], where
// ZS_J is the analytical integral over panel J of the far-field wave factor,
// an edge sum of (CEP(l+1) - CEP(l)) / (ZJ(l+1) - ZJ(l)) terms with
// ZJ(k) = k0 (z_k - i wbar_k), wbar = (x - XEFF) cos(theta) + (y - YEFF) sin(theta),
// CEP = exp(ZJ) and, in finite depth, CEM = exp(-ZJ - 2 k0 h); ZS' is the same
// for the mirror image of the half mesh (y -> -y). One CTA = 128 panels x one
// direction; each thread builds its panel's ZS (and ZS'), multiplies by the
// source strengths of every problem and the CTA reduces them into H.
// The quantities that decide a branch (wbar, ZJ, ZC = ZJ(l+1) - ZJ(l) and the
// depth switches) are rounded exactly in the reference's order.
#pragma once
#include "common.cuh"

namespace nb200 {

constexpr int KOCHIN_THREADS = 128;

NB_HD __forceinline__ void kochin_node(const double* __restrict__ xyz, int k, double kwave, double depth,
                                       double xeff, double yeff, double ct, double st, double ys, cplx& zj,
                                       cplx& cep, cplx& cem) {
  const double x = xyz[3 * k], y = ys * xyz[3 * k + 1], z = xyz[3 * k + 2];
  const double wbar = XADD(XMUL(XSUB(x, xeff), ct), XMUL(XSUB(y, yeff), st));
  zj = mk(XMUL(kwave, z), XMUL(kwave, -wbar));
  cep = (zj.re < -18.) ? mk(0., 0.) : cexp_(zj);
  const double tre = XSUB(-zj.re, XMUL(XMUL(2., kwave), depth));
  const bool off = (tre < -18.) || (-XMUL(kwave, depth) >= 0.);
  cem = off ? mk(0., 0.) : cexp_(mk(tre, -zj.im));
}

// ZS of panel i (and ZS' of its mirror half) for the direction (ct, st)
NB_HD __forceinline__ void kochin_panel(const double* __restrict__ xyz, const int* __restrict__ m1234,
                                        const double* __restrict__ rows, int nfa, int nsymy, double kwave,
                                        double depth, double xeff, double yeff, double ct, double st, int i,
                                        cplx* zs) {
  const int kk[5] = {m1234[4 * i] - 1, m1234[4 * i + 1] - 1, m1234[4 * i + 2] - 1, m1234[4 * i + 3] - 1,
                     m1234[4 * i] - 1};
  const double XN = rows[3 * nfa + i], YN = rows[4 * nfa + i], ZN = rows[5 * nfa + i];
  const double kh = XMUL(kwave, depth);
  for (int half = 0; half <= nsymy; ++half) {
    const double ys = half ? -1. : 1.;
    const cplx ZMS = mk(half ? -YN : YN, -(ZN * st));
    const cplx ZNS = mk(XN, -(ZN * ct));
    cplx zj[5], cep[5], cem[5];
#pragma unroll
    for (int l = 0; l < 4; ++l) kochin_node(xyz, kk[l], kwave, depth, xeff, yeff, ct, st, ys, zj[l], cep[l], cem[l]);
    zj[4] = zj[0]; cep[4] = cep[0]; cem[4] = cem[0];
    cplx acc = mk(0., 0.);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double dx = xyz[3 * kk[l + 1]] - xyz[3 * kk[l]];
      const double dy = xyz[3 * kk[l + 1] + 1] - xyz[3 * kk[l] + 1];
      const cplx ZCS = half ? ZMS * dx + ZNS * dy : ZMS * dx - ZNS * dy;
      const cplx ZC = mk(XSUB(zj[l + 1].re, zj[l].re), XSUB(zj[l + 1].im, zj[l].im));
      cplx ZHS, ZHD;
      if (fabs(ZC.im) < 1.E-04 && fabs(ZC.re) < 1.E-04) {
        ZHS = 0.5 * (cep[l + 1] + cep[l]);
        ZHD = -0.5 * (cem[l + 1] + cem[l]);
      } else {
        ZHS = (cep[l + 1] - cep[l]) / ZC;
        ZHD = (cem[l + 1] - cem[l]) / ZC;
      }
      const cplx a = ZCS * ZHS, b = ZCS * ZHD;
      acc = acc + a + mk(b.re, -b.im);
    }
    const double sgn = half ? -1. : 1.;
    if ((kh > 18.) || (kh <= 0.)) acc = (sgn / kwave) * acc;
    else acc = (sgn * 0.5 * exp(kh) / sinh(kh) / kwave) * acc;
    zs[half] = acc;
  }
}

// out (ntheta x nprob complex) must be zero; zigb/zigs: nprob x nfa complex
__global__ void __launch_bounds__(KOCHIN_THREADS)
    kochin_kernel(const double* __restrict__ xyz, const int* __restrict__ m1234, const double* __restrict__ rows,
                  int nfa, int nsymy, double kwave, double depth, double xeff, double yeff,
                  const double2* __restrict__ cs, int nprob, const double2* __restrict__ zigb,
                  const double2* __restrict__ zigs, int ntheta, double2* out) {
  __shared__ double red[2][KOCHIN_THREADS / 32];
  const int i = blockIdx.x * KOCHIN_THREADS + threadIdx.x;
  const int t = blockIdx.y;
  const double ct = cs[t].x, st = cs[t].y;
  cplx zs[2] = {mk(0., 0.), mk(0., 0.)};
  if (i < nfa) kochin_panel(xyz, m1234, rows, nfa, nsymy, kwave, depth, xeff, yeff, ct, st, i, zs);
  const double q = 0.25 / 3.141592653589793;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int p = 0; p < nprob; ++p) {
    cplx v = mk(0., 0.);
    if (i < nfa) {
      const double2 b = zigb[(long long)p * nfa + i];
      v = mk(b.x, b.y) * zs[0];
      if (nsymy) {
        const double2 s = zigs[(long long)p * nfa + i];
        v = v + mk(s.x, s.y) * zs[1];
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      v.re += __shfl_xor_sync(0xffffffffu, v.re, o);
      v.im += __shfl_xor_sync(0xffffffffu, v.im, o);
    }
    if (lane == 0) {
      red[0][warp] = v.re;
      red[1][warp] = v.im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double re = 0., im = 0.;
      for (int w = 0; w < KOCHIN_THREADS / 32; ++w) {
        re += red[0][w];
        im += red[1][w];
      }
      atomicAdd(&out[t + (long long)ntheta * p].x, q * re);
      atomicAdd(&out[t + (long long)ntheta * p].y, q * im);
    }
    __syncthreads();
  }
}

}  // namespace nb200
