// Free-surface elevation from the solved source strengths
// (COMPUTE_POTENTIAL_DOMAIN.f90:24-82 with COMPUTE_GREEN_FREESURFACE.f90, as
// called at SOLVE_BEM.f90:104-109): at field points (x, y, 0)
//   PHI = sum_J [ZIGB(J), ZIGS(J)] combined with the single-layer Green values
//   SP1, SP2, SM1, SM2 at the field point, and ETA = i W / G PHI.
// The field-point Green functions are the collocation ones with the point not
// clipped to ZER and no self term (VVV, with DHSL = 2 Depth for both forms),
// always the tabulated wave branch (VNV, VNVF), and in finite depth the last
// exponential image replaced by the exact panel integral at the point's
// mirror image (VVG). One thread per field point; the panels are split over
// blockIdx.y and the partial potentials of every problem summed with atomics.
#pragma once
#include "assembly.cuh"

namespace nb200 {

// VVG (COMPUTE_GREEN_FREESURFACE.f90:911-997), single-layer part: exact
// integral over panel P (reflection JJ) at (XPO, YPO, ZPO); the reference's
// literal 12.5663706 for 4 pi is kept
NB_HD __noinline__ double vvg_fs(const PanelRec& P, int JJ, double XPO, double YPO, double ZPO) {
  const int MJJ = (JJ & 1) ? 1 : -1;
  const double dx = XSUB(XPO, P.xg), dy = XSUB(YPO, P.yg * MJJ), dz = XSUB(ZPO, P.zg);
  const double RO = XSQRT(XADD(XADD(XMUL(dx, dx), XMUL(dy, dy)), XMUL(dz, dz)));
  const double GZ = XADD(XADD(XMUL(dx, P.xn), XMUL(XMUL(dy, P.yn), (double)MJJ)), XMUL(dz, P.zn));
  if (XSUB(RO, XMUL(7., P.tdis)) > 0.) return -P.aire / (RO * 12.5663706);
  double RR[5], XL[5], YL[5], ZL[5];
  for (int L = 0; L < 4; ++L) {
    XL[L] = P.vx[L]; YL[L] = P.vy[L]; ZL[L] = P.vz[L];
    const double ax = XPO - XL[L], ay = YPO - YL[L] * MJJ, az = ZPO - ZL[L];
    RR[L] = sqrt(ax * ax + ay * ay + az * az);
  }
  XL[4] = XL[0]; YL[4] = YL[0]; ZL[4] = ZL[0]; RR[4] = RR[0];
  const double AGZ = fabs(GZ);
  double FS = 0.;
  for (int L = 0; L < 4; ++L) {
    const double ex = XSUB(XL[L + 1], XL[L]), ey = XSUB(YL[L + 1], YL[L]), ez = XSUB(ZL[L + 1], ZL[L]);
    const double DK = XSQRT(XADD(XADD(XMUL(ex, ex), XMUL(ey, ey)), XMUL(ez, ez)));
    if (XSUB(DK, XMUL(1.E-3, P.tdis)) <= 0.) continue;
    const double PJ = ex / DK, QJ = ey / DK * MJJ, RJ = ez / DK;
    const double GYX = MJJ * P.yn * RJ - P.zn * QJ;
    const double GYY = P.zn * PJ - P.xn * RJ;
    const double GYZ = P.xn * QJ - P.yn * MJJ * PJ;
    const double GY = (XPO - XL[L]) * GYX + (YPO - YL[L] * MJJ) * GYY + (ZPO - ZL[L]) * GYZ;
    const double DDK = 2. * DK, ANT = GY * DDK, RS = RR[L + 1] + RR[L];
    const double DNT = RS * RS - DK * DK + 2. * AGZ * RS;
    const double ANL = RS + DK, DNL = RS - DK;
    const double AT = (AGZ >= XMUL(1.E-4, P.tdis)) ? atan(ANT / DNT) : 0.;
    FS += GY * log(ANL / DNL) - 2. * AGZ * AT;
  }
  return FS * (-MJJ / 12.5663706);
}

// single-layer values of panel P at a field point (XPO, YPO, ZPO)
template <bool FD>
NB_HD __forceinline__ void field_green(const GreenCtx& g, const OmegaParams& om, double XPO, double YPO,
                                            double ZPO, const PanelRec& P, double& SP1, double& SP2, double& SM1,
                                            double& SM2) {
  const int NJJ = g.nsymy + 1;
  RankineOut r;
  rankine<FD>(g, XMUL(2., om.h), XPO, YPO, ZPO, false, P, r, false);
  WaveJJ w[2];
  w[1] = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
  if (FD) {
    wave_fd_pair(g, om, XPO, YPO, ZPO, P, NJJ, w);
    // exponential images (VNVF image loop), the last term's second image by VVG
    const double QPI = 4. * 3.141592653589793;
    const double H = om.h, H2 = XMUL(2., H), H4 = XMUL(4., H);
    const double ACT = -0.5 * P.aire / QPI;
    const int nexp1 = om.nexp + 1;
#pragma unroll 1
    for (int b = 0; b < NJJ; ++b) {
      const double dx = XSUB(XPO, P.xg), dy = XSUB(YPO, P.yg * (b ? -1. : 1.));
      const double R = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
      const double r2 = XMUL(R, R);
      double fs = 0.;
#pragma unroll 1
      for (int KE = 1; KE <= nexp1; ++KE) {
        const double AQT = ACT * om.ar[KE];
        const double HA = XMUL(H, om.ambda[KE]);
        double zp[4];
        zp[0] = XSUB(XADD(XSUB(ZPO, H2), HA), P.zg);
        zp[1] = XSUB(XSUB(-ZPO, HA), P.zg);
        zp[2] = XSUB(XADD(XSUB(-ZPO, H4), HA), P.zg);
        zp[3] = XSUB(XSUB(XADD(ZPO, H2), HA), P.zg);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k == 1 && KE == nexp1) {
            fs += vvg_fs(P, b + 1, XPO, YPO, -ZPO);
            continue;
          }
          const double RRk = XADD(r2, XMUL(zp[k], zp[k]));
          if (RRk > g.ro_eps2) fs += AQT * rsqrt(RRk);
        }
      }
      w[b].FS1 += fs;
    }
  } else {
    wave_infd_pair(g, om, XPO, YPO, ZPO, P, NJJ, w);
  }
  double s1 = 1., s2 = 1.;
  if (!FD) {
    const double DPI = 2. * 3.141592653589793, DPI2 = 2. * 3.141592653589793 * 3.141592653589793;
    const double AKAIR = om.k0 * P.aire;
    s1 = -AKAIR / DPI2;
    s2 = -AKAIR / DPI;
  }
  const double BM = (NJJ == 2) ? -1. : 1.;
  SP1 = r.FSP + (w[0].FS1 + w[1].FS1) * s1;
  SM1 = r.FSM + (w[0].FS1 + BM * w[1].FS1) * s1;
  SP2 = (w[0].FS2 + w[1].FS2) * s2;
  SM2 = (w[0].FS2 + BM * w[1].FS2) * s2;
}

constexpr int FS_POINTS = 128;
constexpr int FS_PANELS = 128;
constexpr int FS_MAXP = 16;

// phi (npts x nprob complex, zeroed) += potential of the panels of chunk blockIdx.y
template <bool FD>
__global__ void __launch_bounds__(FS_POINTS)
    freesurface_kernel(GreenCtx g, const OmegaParams* __restrict__ omp, const PanelRec* __restrict__ rec, int nfa,
                       const double2* __restrict__ xy, int npts, int nprob, const double2* __restrict__ zigb,
                       const double2* __restrict__ zigs, double2* phi) {
  __shared__ PanelRec sp[ASM_TJ];
  __shared__ OmegaParams som;
  stage_params(omp, &som);
  const int q = blockIdx.x * FS_POINTS + threadIdx.x;
  const double XPO = q < npts ? xy[q].x : 0., YPO = q < npts ? xy[q].y : 0.;
  double pot1[FS_MAXP], pot2[FS_MAXP];
#pragma unroll
  for (int p = 0; p < FS_MAXP; ++p) pot1[p] = pot2[p] = 0.;
  const int jbeg = blockIdx.y * FS_PANELS, jend = min(nfa, jbeg + FS_PANELS);
  for (int j0 = jbeg; j0 < jend; j0 += ASM_TJ) {
    const int nj = min(ASM_TJ, jend - j0);
    __syncthreads();
    stage_panels(rec, j0, nj, sp);
    __syncthreads();
    if (q >= npts) continue;
#pragma unroll 1
    for (int jj = 0; jj < nj; ++jj) {
      double SP1, SP2, SM1, SM2;
      field_green<FD>(g, som, XPO, YPO, 0., sp[jj], SP1, SP2, SM1, SM2);
      const int J = j0 + jj;
#pragma unroll
      for (int p = 0; p < FS_MAXP; ++p) {
        if (p >= nprob) break;
        const double2 b = zigb[(long long)p * nfa + J];
        if (g.nsymy == 0) {
          pot1[p] += b.x * SP1 - b.y * SP2;
          pot2[p] += b.x * SP2 + b.y * SP1;
        } else {
          const double2 s = zigs[(long long)p * nfa + J];
          const double C1 = b.x * (SP1 + SM1) + s.x * (SP1 - SM1), D1 = b.y * (SP2 + SM2) + s.y * (SP2 - SM2);
          const double C2 = b.x * (SP2 + SM2) + s.x * (SP2 - SM2), D2 = b.y * (SP1 + SM1) + s.y * (SP1 - SM1);
          pot1[p] += (C1 - D1) * 0.5;
          pot2[p] += (C2 + D2) * 0.5;
        }
      }
    }
  }
  if (q >= npts) return;
#pragma unroll
  for (int p = 0; p < FS_MAXP; ++p) {
    if (p >= nprob) break;
    atomicAdd(&phi[q + (long long)npts * p].x, pot1[p]);
    atomicAdd(&phi[q + (long long)npts * p].y, pot2[p]);
  }
}

}  // namespace nb200
