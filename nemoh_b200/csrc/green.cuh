// Device Green functions of the Nemoh BEM solve (sm_100a, FP64).
//
// Per pair (collocation panel I, source panel J) this evaluates what the
// reference computes in
//   VAVINFD / VAVFD   (Solver/Core/COMPUTE_GREEN_INFD.f90:33-220,
//                      Solver/Core/COMPUTE_GREEN_FD.f90:32-219)   Rankine part
//   VNSINFD / VNSFD   (COMPUTE_GREEN_INFD.f90:223-503,
//                      COMPUTE_GREEN_FD.f90:222-868)               wave part
// and returns both symmetry classes at once: the normal-derivative entries
// D+ = grad G+ . n_I and D- = grad G- . n_I (the ZIJ fill of
// SOLVE_BEM_INFD_DIRECT.f90:84-104) and the single-layer entries S+ = (SP1,SP2),
// S- = (SM1,SM2) used for the boundary potential (:154-163).
//
// Branch-deciding quantities use the exactly rounded X* macros (common.cuh).
#pragma once
#include "common.cuh"

namespace nb200 {

struct GreenCtx {
  double ro_eps2;                   // largest x with sqrt(x) <= 1e-4 (exact RO > EPS test on RO^2)
  const double* xr;                 // XR(1..328) at [1..328]
  const double* xz;                 // XZ(1..46) at [1..46]
  const double4* apd;               // {APD1X, APD1Z, APD2X, APD2Z}(I,J) at (I-1)+328*(J-1)
  const StencilThresholds* thr;
  double zer;                       // ZER (PREPARE_MESH.f90:58-69)
  int nsymy;
  int* status;                      // device status word (first error wins)
};

struct PairOut {
  double dp_re, dp_im, dm_re, dm_im;  // D+, D-
  double sp_re, sp_im, sm_re, sm_im;  // S+, S-
};

__device__ __forceinline__ void set_status(int* st, int code) { atomicCAS(st, 0, code); }

// --- GG(Z,CEX): ELEMENTARY_FNS.f90:31-81 ----------------------------------
__device__ __noinline__ cplx GG(cplx Z, cplx CEX) {
  const cplx IPI = mk(0., 3.14159265);
  if (Z.re + 16. <= 0.) {
    cplx Y = 1. / Z;
    return Y * (1. + Y * (-1. + Y * (2. + Y * (-6. + Y * (24. + Y * (-120.))))));
  }
  double T = Z.im;
  cplx G;
  if (fabs(T) - 10. > 0.) {
    G = 0.711093 / (Z + 0.415775) + 0.278518 / (Z + 2.29428) + 0.010389 / (Z + 6.2900);
    return (T < 0.) ? G - IPI * CEX : G + IPI * CEX;
  }
  if (Z.re + 0.5 > 0.) {
    cplx num = clog_(Z) * (1. + Z * (0.23721365E+00 + Z * (0.206543E-01 + Z * (0.763297E-03 +
               Z * 0.97087007E-05)))) + 0.5772156649E+00 * (0.99999207E+00 +
               Z * (-0.149545886E+01 + Z * (0.41806426E-01 + Z * (-0.3000591E-01 +
               Z * (0.19387339E-02 + Z * (-0.51801555E-03))))));
    cplx den = 1. + Z * (-0.76273617E+00 + Z * (0.28388363E+00 + Z * (-0.66786033E-01 + Z * (0.12982719E-01
               + Z * (-0.8700861E-03 + Z * 0.2989204E-03)))));
    G = -(num / den);
    return (T < 0.) ? G - IPI * CEX : G + IPI * CEX;
  }
  const double s = (T < 0.) ? 1. : -1.;   // conjugate coefficients in the upper half plane
  cplx num = ((((((mk(1.000000, s * 1.3935496E-06) * Z + mk(15.82958, -s * 20.14222))
      * Z + mk(-70.52863, -s * 227.9511)) * Z + mk(-985.4221, -s * 226.6272)) * Z
      + mk(-1202.318, s * 1580.907)) * Z + mk(953.2441, s * 1342.447)) * Z
      + mk(417.3716, -s * 196.6665)) * Z + mk(-9.881266, -s * 24.24952);
  cplx den = (((((((mk(1.000000, 0.0) * Z + mk(16.83184, -s * 20.14481)) * Z
      + mk(-55.66969, -s * 248.1167)) * Z + mk(-1068.640, -s * 434.4707)) * Z
      + mk(-2082.250, s * 1522.471)) * Z + mk(383.3455, s * 2730.378)) * Z
      + mk(1216.791, s * 351.7189)) * Z + mk(115.3926, -s * 161.2647)) * Z
      + mk(-3.777369, -s * 4.510900);
  return (T < 0.) ? num / den - IPI * CEX : num / den + IPI * CEX;
}

// COMPUTE_GREEN_INFD.f90:641-645
__device__ __forceinline__ double PL2(double U1, double U2, double U3, double XU) {
  return ((XU - U1) * (XU - U2)) / ((U3 - U1) * (U3 - U2));
}

// integer part of a monotone log10 expression, made exact by thresholds
__device__ __forceinline__ int stencil_adjust(double x, const double* thr, int k) {
  k = max(0, min(k, 47));
#pragma unroll 1
  for (int it = 0; it < 4 && k < 47 && x >= __ldg(thr + k + 1); ++it) ++k;
#pragma unroll 1
  for (int it = 0; it < 4 && k > 0 && x < __ldg(thr + k); ++it) --k;
  return k;
}

// KJ of COMPUTE_GREEN_INFD.f90:292-298 (AKZ in (-16, -1.5e-6])
__device__ __forceinline__ int stencil_kj(double AKZ, const StencilThresholds* T) {
  double x = -AKZ;
  int k;
  if (AKZ < -1.E-2) k = stencil_adjust(x, T->kj8, (int)(8. * (log10(x) + 4.5)));
  else k = stencil_adjust(x, T->kj5, (int)(5. * (log10(x) + 6.)));
  k = max(k, 2);
  return min(k, 45);
}

// KI of COMPUTE_GREEN_INFD.f90:299-305
__device__ __forceinline__ int stencil_ki(double AKR, const StencilThresholds* T) {
  int k;
  if (AKR < 1.) {
    double y = XADD(AKR, 1.E-20);
    k = stencil_adjust(y, T->ki5, (int)(5. * (log10(y) + 6.) + 1.));
  } else {
    k = (int)XADD(XMUL(3., AKR), 28.);
  }
  k = max(k, 2);
  return min(k, 327);
}

struct Lagrange {
  int KI, KJ;
  double XL1, XL2, XL3, ZL1, ZL2, ZL3;
};

__device__ __forceinline__ void lagrange_x(const GreenCtx& g, double AKR, Lagrange& L) {
  L.KI = stencil_ki(AKR, g.thr);
  double a = __ldg(g.xr + L.KI - 1), b = __ldg(g.xr + L.KI), c = __ldg(g.xr + L.KI + 1);
  L.XL1 = PL2(b, c, a, AKR);
  L.XL2 = PL2(c, a, b, AKR);
  L.XL3 = PL2(a, b, c, AKR);
}
__device__ __forceinline__ void lagrange_z(const GreenCtx& g, double AKZ, Lagrange& L) {
  L.KJ = stencil_kj(AKZ, g.thr);
  double a = __ldg(g.xz + L.KJ - 1), b = __ldg(g.xz + L.KJ), c = __ldg(g.xz + L.KJ + 1);
  L.ZL1 = PL2(b, c, a, AKZ);
  L.ZL2 = PL2(c, a, b, AKZ);
  L.ZL3 = PL2(a, b, c, AKZ);
}

__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// 3x3 Lagrange interpolation of the four tables (:306-319, :345-352)
__device__ __forceinline__ double4 interp4(const GreenCtx& g, const Lagrange& L) {
  double4 r = make_double4(0., 0., 0., 0.);
  const double zl[3] = {L.ZL1, L.ZL2, L.ZL3};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const double4* row = g.apd + (L.KI - 2) + TAB_IR * (L.KJ - 2 + b);
    double4 t1 = ldg4(row), t2 = ldg4(row + 1), t3 = ldg4(row + 2);
    double4 F;
    F.x = L.XL1 * t1.x + L.XL2 * t2.x + L.XL3 * t3.x;
    F.y = L.XL1 * t1.y + L.XL2 * t2.y + L.XL3 * t3.y;
    F.z = L.XL1 * t1.z + L.XL2 * t2.z + L.XL3 * t3.z;
    F.w = L.XL1 * t1.w + L.XL2 * t2.w + L.XL3 * t3.w;
    r.x += zl[b] * F.x;
    r.y += zl[b] * F.y;
    r.z += zl[b] * F.z;
    r.w += zl[b] * F.w;
  }
  return r;  // {PD1X, PD1Z, PD2X, PD2Z}
}

// --- Rankine part: VAVINFD (DH=0, KKK=1) / VAVFD (DH=2h, KKK=2) ----------
struct RankineOut {
  double FSP, FSM, VSXP, VSYP, VSZP, VSXM, VSYM, VSZM;
};

// exact edge-sum panel integral and gradient for one image (:99-174)
__device__ __noinline__ void rankine_near(double XOI, double YOI, double ZOI, const PanelRec& P, int MY, int MZ,
                                          double DHMH, double& AIJS, double& VXS, double& VYS, double& VZS) {
  double TXN[5], TYN[5], TZN[5], RR[5], DRX[5], DRY[5], DRZ[5];
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    TXN[L] = P.vx[L];
    TYN[L] = P.vy[L] * MY;
    TZN[L] = XSUB(P.vz[L] * MZ, DHMH);
  }
  TXN[4] = TXN[0]; TYN[4] = TYN[0]; TZN[4] = TZN[0];
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    double dx = XOI - TXN[L], dy = YOI - TYN[L], dz = ZOI - TZN[L];
    RR[L] = sqrt(dx * dx + dy * dy + dz * dz);
    double inv = 1. / RR[L];
    DRX[L] = dx * inv;
    DRY[L] = dy * inv;
    DRZ[L] = dz * inv;
  }
  RR[4] = RR[0]; DRX[4] = DRX[0]; DRY[4] = DRY[0]; DRZ[4] = DRZ[0];
  const double A3J = P.xn, A6J = P.yn * MY, A9J = P.zn * MZ;
  const double ZOJ = XSUB(P.zg * MZ, DHMH);
  const double GZ = XADD(XADD(XMUL(XSUB(XOI, P.xg), A3J), XMUL(XSUB(YOI, P.yg * MY), A6J)),
                         XMUL(XSUB(ZOI, ZOJ), A9J));
  const double AGZ = fabs(GZ);
  const double SGN = copysign(1., GZ);
  const double dklim = XMUL(1.E-3, P.tdis), gzlim = XMUL(1.E-4, P.tdis);
  AIJS = 0.; VXS = 0.; VYS = 0.; VZS = 0.;
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    double ex = XSUB(TXN[L + 1], TXN[L]), ey = XSUB(TYN[L + 1], TYN[L]), ez = XSUB(TZN[L + 1], TZN[L]);
    double DK = XSQRT(XADD(XADD(XMUL(ex, ex), XMUL(ey, ey)), XMUL(ez, ez)));
    if (DK >= dklim) {
      double idk = 1. / DK;
      double PJ = ex * idk, QJ = ey * idk, RJ = ez * idk;
      double GYX = A6J * RJ - A9J * QJ;
      double GYY = A9J * PJ - A3J * RJ;
      double GYZ = A3J * QJ - A6J * PJ;
      double GY = (XOI - TXN[L]) * GYX + (YOI - TYN[L]) * GYY + (ZOI - TZN[L]) * GYZ;
      double DDK = 2. * DK;
      double ANT = GY * DDK;
      double RS = RR[L + 1] + RR[L];
      double DNT = RS * RS - DK * DK + 2. * AGZ * RS;
      double ANL = RS + DK;
      double DNL = RS - DK;
      double ALDEN = log(ANL / DNL);
      double AT = (AGZ >= gzlim) ? atan(ANT / DNT) : 0.;
      AIJS += GY * ALDEN - 2. * AGZ * AT;
      double DAT = 2. * AT * SGN;
      double ANLX = DRX[L + 1] + DRX[L], ANLY = DRY[L + 1] + DRY[L], ANLZ = DRZ[L + 1] + DRZ[L];
      double DR = 2. * (RS + AGZ);
      double DS = 2. * RS * SGN;
      double DENT = ANT * ANT + DNT * DNT;
      double iDENT = 1. / DENT;
      double ATX = (GYX * DDK * DNT - (DR * ANLX + A3J * DS) * ANT) * iDENT;
      double ATY = (GYY * DDK * DNT - (DR * ANLY + A6J * DS) * ANT) * iDENT;
      double ATZ = (GYZ * DDK * DNT - (DR * ANLZ + A9J * DS) * ANT) * iDENT;
      double DLOGG = (DNL - ANL) / (ANL * DNL);
      VXS += GYX * ALDEN + GY * ANLX * DLOGG - 2. * AGZ * ATX - DAT * A3J;
      VYS += GYY * ALDEN + GY * ANLY * DLOGG - 2. * AGZ * ATY - DAT * A6J;
      VZS += GYZ * ALDEN + GY * ANLZ * DLOGG - 2. * AGZ * ATZ - DAT * A9J;
    }
  }
}

template <bool FD>
__device__ __forceinline__ void rankine(const GreenCtx& g, double DH, double XGI, double YGI, double ZGI, bool self,
                                        const PanelRec& P, RankineOut& o) {
  const double QPI = 4. * 3.141592653589793;
  const double DPI = 2. * 3.141592653589793;
  const int NJJ = 2 * (g.nsymy + 1);
  const double MK = FD ? -1. : 1.;
  double XOI = XGI, YOI = YGI, ZOI = ZGI;
  if (ZGI > g.zer) ZOI = FD ? XMUL(20., g.zer) : g.zer;
  double AIJS[4], VXS[4], VYS[4], VZS[4];
  const double lim7 = XMUL(7., P.tdis);
#pragma unroll
  for (int JJ = 1; JJ <= 4; ++JJ) {
    if (JJ > NJJ) break;
    const int MJJ = (JJ & 1) ? 1 : -1;
    const int MY = (JJ >= 3) ? -1 : 1;
    const int MZ = (JJ == 2 || JJ == 3) ? -1 : 1;
    const double DHMH = (JJ == 2 || JJ == 3) ? DH : 0.;
    const double XOJ = P.xg, YOJ = P.yg * MY, ZOJ = XSUB(P.zg * MZ, DHMH);
    const double dx = XSUB(XOI, XOJ), dy = XSUB(YOI, YOJ), dz = XSUB(ZOI, ZOJ);
    const double RO = XSQRT(XADD(XADD(XMUL(dx, dx), XMUL(dy, dy)), XMUL(dz, dz)));
    double a, vx, vy, vz;
    if (RO > lim7) {
      a = P.aire / RO;
      double ASRO = a / (RO * RO);
      vx = -dx * ASRO;
      vy = -dy * ASRO;
      vz = -dz * ASRO;
    } else {
      rankine_near(XOI, YOI, ZOI, P, MY, MZ, DHMH, a, vx, vy, vz);
      if (self && JJ == 1) {
        vx -= DPI * P.xn;
        vy -= DPI * (P.yn * MY);
        vz -= DPI * (P.zn * MZ);
      } else {
        a *= MJJ; vx *= MJJ; vy *= MJJ; vz *= MJJ;
      }
    }
    AIJS[JJ - 1] = a; VXS[JJ - 1] = vx; VYS[JJ - 1] = vy; VZS[JJ - 1] = vz;
  }
  const double iq = -1. / QPI;
  if (g.nsymy == 1) {
    o.FSP = (AIJS[0] - MK * (AIJS[1] + AIJS[2]) + AIJS[3]) * iq;
    o.FSM = (AIJS[0] - MK * (AIJS[1] - AIJS[2]) - AIJS[3]) * iq;
    o.VSXP = (VXS[0] - MK * (VXS[1] + VXS[2]) + VXS[3]) * iq;
    o.VSYP = (VYS[0] - MK * (VYS[1] + VYS[2]) + VYS[3]) * iq;
    o.VSZP = (VZS[0] - MK * (VZS[1] + VZS[2]) + VZS[3]) * iq;
    o.VSXM = (VXS[0] - MK * (VXS[1] - VXS[2]) - VXS[3]) * iq;
    o.VSYM = (VYS[0] - MK * (VYS[1] - VYS[2]) - VYS[3]) * iq;
    o.VSZM = (VZS[0] - MK * (VZS[1] - VZS[2]) - VZS[3]) * iq;
  } else {
    o.FSP = o.FSM = (AIJS[0] - MK * AIJS[1]) * iq;
    o.VSXP = o.VSXM = (VXS[0] - MK * VXS[1]) * iq;
    o.VSYP = o.VSYM = (VYS[0] - MK * VYS[1]) * iq;
    o.VSZP = o.VSZM = (VZS[0] - MK * VZS[1]) * iq;
  }
}

// per-reflection wave contributions (FS1..VSZ2 of one JJ)
struct WaveJJ {
  double FS1, FS2, VSX1, VSY1, VSZ1, VSX2, VSY2, VSZ2;
};

// --- VNSINFD free-surface-panel branch (COMPUTE_GREEN_INFD.f90:385-453) ---
__device__ __noinline__ void wave_infd_fs(const OmegaParams& om, double XGI, double YGI, double ZMIII, int BX,
                                          const PanelRec& P, WaveJJ& w) {
  const double EPS = 0.0001;
  const double AK0 = om.k0;
  w = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
  for (int IT = 1; IT <= om.nq; ++IT) {
    const double CT = om.ct[IT], ST = om.st[IT];
    cplx Z[5], CEX[5], GZ[5];
    for (int L = 0; L < 4; ++L) {
      double re = XMUL(AK0, XADD(ZMIII, P.vz[L]));
      double im = XMUL(AK0, XADD(XMUL(XSUB(XGI, P.vx[L]), CT), XMUL(XSUB(YGI, P.vy[L] * BX), ST)));
      Z[L] = mk(re, im);
      CEX[L] = (re > -25.) ? cexp_(Z[L]) : mk(0., 0.);
      GZ[L] = GG(Z[L], CEX[L]);
    }
    Z[4] = Z[0]; CEX[4] = CEX[0]; GZ[4] = GZ[0];
    cplx ZA = mk(0, 0), ZB = mk(0, 0), ZVS = mk(0, 0);
    for (int L = 0; L < 4; ++L) {
      cplx C1 = mk(XSUB(Z[L + 1].re, Z[L].re), XSUB(Z[L + 1].im, Z[L].im));
      cplx ASD, BSD, CSD;
      if (fabs(C1.im) < EPS && fabs(C1.re) < EPS) {
        ASD = (GZ[L + 1] + GZ[L]) * 0.5;
        BSD = (CEX[L + 1] + CEX[L]) * 0.5;
        CSD = ASD - (0.5 / Z[L + 1] + 0.5 / Z[L]);
      } else {
        CSD = (GZ[L + 1] - GZ[L]) / C1;
        ASD = (GZ[L + 1] - GZ[L] + clog_(Z[L + 1] / Z[L])) / C1;
        BSD = (CEX[L + 1] - CEX[L]) / C1;
      }
      cplx C2 = mk(P.yn * BX, -P.zn * ST) * (P.vx[(L + 1) & 3] - P.vx[L]) -
                mk(P.xn, -P.zn * CT) * ((P.vy[(L + 1) & 3] - P.vy[L]) * BX);
      ZA = ZA + ASD * C2;
      ZB = ZB + BSD * C2;
      ZVS = ZVS + CSD * C2;
    }
    const double cq = om.cq[IT];
    w.FS1 += cq * ZA.re;
    w.FS2 += cq * ZB.re;
    w.VSX1 -= cq * CT * ZVS.im;
    w.VSX2 -= cq * CT * ZB.im;
    w.VSY1 -= cq * ST * ZVS.im;
    w.VSY2 -= cq * ST * ZB.im;
    w.VSZ1 += cq * ZVS.re;
    w.VSZ2 += cq * ZB.re;
  }
  const double s = BX / (AK0 * P.aire);
  w.FS1 *= s; w.FS2 *= s; w.VSX1 *= s; w.VSX2 *= s; w.VSY1 *= s; w.VSY2 *= s; w.VSZ1 *= s; w.VSZ2 *= s;
}

// --- VNSINFD tabulated branch for one reflection BX (:271-382) -------------
__device__ __forceinline__ void wave_infd_jj(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI,
                                             double ZMIII, int BX, const PanelRec& P, WaveJJ& w) {
  const double PI = 3.141592653589793, PI4 = 0.7853981633974483, DPI = 2. * PI, EPS = 0.0001;
  const double AK0 = om.k0;
  const double YMJJJ = P.yg * BX;
  const double dx = XSUB(XGI, P.xg), dy = XSUB(YGI, YMJJJ);
  const double RRR = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
  const double AKR = XMUL(AK0, RRR);
  const double ZZZ = XADD(ZMIII, P.zg);
  const double AKZ = XMUL(AK0, ZZZ);
  const double DD = XSQRT(XADD(XMUL(RRR, RRR), XMUL(ZZZ, ZZZ)));
  double PSURR = 0.;
  if (DD > EPS) {
    double t = AK0 * DD;
    PSURR = PI / (t * t * t);
  }
  double PD1Z, PD2Z, VZ1, VZ2, PD1X = 0., PD2X = 0., VR1 = 0., VR2 = 0.;
  if (AKZ > -1.5E-6) {
    set_status(g.status, ST_AKZ_UNDEFINED);
    w = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
    return;
  }
  if (AKZ > -16.) {
    if (AKR < 99.7) {
      Lagrange L;
      lagrange_x(g, AKR, L);
      lagrange_z(g, AKZ, L);
      double4 t = interp4(g, L);
      PD1X = t.x; PD1Z = t.y; PD2X = t.z; PD2Z = t.w;
    } else {
      double EPZ = exp(AKZ);
      double SQ = sqrt(DPI / AKR);
      double SIK, CSK;
      sincos(AKR - PI4, &SIK, &CSK);
      PD1Z = PSURR * AKZ - PI * EPZ * SQ * SIK;
      PD2Z = EPZ * SQ * CSK;
      double DSK = 0.5 / AKR;
      PD1X = -PSURR * AKR + PI * EPZ * SQ * (CSK - DSK * SIK);
      PD2X = EPZ * SQ * (SIK + DSK * CSK);
    }
    VZ1 = PD1Z - PSURR * AKZ;
    VZ2 = PD2Z;
    VR1 = -PD1X - PSURR * AKR;
    VR2 = -PD2X;
  } else {
    PD1Z = PSURR * AKZ;
    PD2Z = 0.;
    VZ1 = 0.;
    VZ2 = 0.;
  }
  w.FS1 = PD1Z;
  w.FS2 = PD2Z;
  if (RRR > EPS) {
    const double iR = 1. / RRR;
    const double CVX = dx * iR, CVY = dy * iR;
    w.VSX1 = VR1 * CVX;
    w.VSX2 = VR2 * CVX;
    w.VSY1 = VR1 * CVY;
    w.VSY2 = VR2 * CVY;
  } else {
    w.VSX1 = w.VSX2 = w.VSY1 = w.VSY2 = 0.;
  }
  w.VSZ1 = VZ1;
  w.VSZ2 = VZ2;
}

// --- VSD: exact Rankine panel integral used by the FD free-surface branch --
// (COMPUTE_GREEN_FD.f90:1514-1609)
__device__ __noinline__ void vsd(const PanelRec& P, int JJ, double XGI, double YGI, double ZIG, double& FS, double& VX,
                                 double& VY, double& VZ) {
  const double QPI = 4. * 4. * atan(1.);
  const int MJJ = (JJ & 1) ? 1 : -1;
  const double QMP = MJJ / (2 * QPI);
  const double dx = XSUB(XGI, P.xg), dy = XSUB(YGI, P.yg * MJJ), dz = XSUB(ZIG, P.zg);
  const double RO = XSQRT(XADD(XADD(XMUL(dx, dx), XMUL(dy, dy)), XMUL(dz, dz)));
  const double YNF = P.yn * MJJ;
  const double GZ = XADD(XADD(XMUL(dx, P.xn), XMUL(dy, YNF)), XMUL(dz, P.zn));
  if (RO > XMUL(7., P.tdis)) {
    FS = -P.aire / (RO * 2 * QPI);
    double ASRO = FS / (RO * RO);
    VX = -dx * ASRO;
    VY = -dy * ASRO;
    VZ = -dz * ASRO;
    return;
  }
  double RR[5], DRX[5], DRY[5], DRZ[5], XF[5], YF[5], ZF[5];
  for (int L = 0; L < 4; ++L) {
    XF[L] = P.vx[L]; YF[L] = P.vy[L]; ZF[L] = P.vz[L];
    double ax = XGI - XF[L], ay = YGI - YF[L] * MJJ, az = ZIG - ZF[L];
    RR[L] = sqrt(ax * ax + ay * ay + az * az);
    DRX[L] = ax / RR[L];
    DRY[L] = ay / RR[L];
    DRZ[L] = az / RR[L];
  }
  XF[4] = XF[0]; YF[4] = YF[0]; ZF[4] = ZF[0];
  RR[4] = RR[0]; DRX[4] = DRX[0]; DRY[4] = DRY[0]; DRZ[4] = DRZ[0];
  double AIJS = 0., VXS = 0., VYS = 0., VZS = 0.;
  const double AGZ = fabs(GZ), SGN = copysign(1., GZ);
  for (int L = 0; L < 4; ++L) {
    double ex = XSUB(XF[L + 1], XF[L]), ey = XSUB(YF[L + 1], YF[L]), ez = XSUB(ZF[L + 1], ZF[L]);
    double DK = XSQRT(XADD(XADD(XMUL(ex, ex), XMUL(ey, ey)), XMUL(ez, ez)));
    if (DK >= XMUL(1.E-3, P.tdis)) {
      double PJ = ex / DK, QJ = ey * MJJ / DK, RJ = ez / DK;
      double GYX = YNF * RJ - P.zn * QJ;
      double GYY = P.zn * PJ - P.xn * RJ;
      double GYZ = P.xn * QJ - YNF * PJ;
      double GY = (XGI - XF[L]) * GYX + (YGI - YF[L] * MJJ) * GYY + (ZIG - ZF[L]) * GYZ;
      double DDK = 2. * DK, ANT = GY * DDK, RS = RR[L + 1] + RR[L];
      double DNT = RS * RS - DK * DK + 2. * AGZ * RS;
      double ANL = RS + DK, DNL = RS - DK;
      double ALDEN = log(ANL / DNL);
      double AT = (AGZ > XMUL(1.E-4, P.tdis)) ? atan(ANT / DNT) : 0.;
      AIJS += GY * ALDEN - 2. * AGZ * AT;
      double DAT = 2. * AT * SGN;
      double ANLX = DRX[L + 1] + DRX[L], ANLY = DRY[L + 1] + DRY[L], ANLZ = DRZ[L + 1] + DRZ[L];
      double DR = 2. * (RS + AGZ), DS = 2. * RS * SGN;
      double DENT = ANT * ANT + DNT * DNT;
      double ATX = (GYX * DDK * DNT - (DR * ANLX + P.xn * DS) * ANT) / DENT;
      double ATY = (GYY * DDK * DNT - (DR * ANLY + YNF * DS) * ANT) / DENT;
      double ATZ = (GYZ * DDK * DNT - (DR * ANLZ + P.zn * DS) * ANT) / DENT;
      double DLG = (DNL - ANL) / (ANL * DNL);
      VXS += GYX * ALDEN + GY * ANLX * DLG - 2. * AGZ * ATX - DAT * P.xn;
      VYS += GYY * ALDEN + GY * ANLY * DLG - 2. * AGZ * ATY - DAT * YNF;
      VZS += GYZ * ALDEN + GY * ANLZ * DLG - 2. * AGZ * ATZ - DAT * P.zn;
    }
  }
  FS = -AIJS * QMP;
  VX = -VXS * QMP;
  VY = -VYS * QMP;
  VZ = -VZS * QMP;
}

// --- VNSFD free-surface-panel branch (COMPUTE_GREEN_FD.f90:707-826) -------
// The theta sum of this branch carries the weights CQ that SOLVE_BEM_FD_DIRECT
// zeroed while CINT_FD filled only its local copies (COMPUTE_GREEN_FD.f90:874),
// so it contributes exactly zero and is skipped; the exponential images (VSD)
// carry the whole term.
__device__ __noinline__ void wave_fd_fs(const OmegaParams& om, double XGI, double YGI, double ZMIII, int JJ,
                                        const PanelRec& P, WaveJJ& w) {
  const double H = om.h;
  w = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
  const double ZP1 = -ZMIII, ZP2 = XADD(ZMIII, XMUL(2., H)), ZP3 = XSUB(ZMIII, XMUL(2., H));
  const double ZP4 = XSUB(-ZMIII, XMUL(4., H));
  for (int KE = 1; KE <= om.nexp + 1; ++KE) {
    const double HA = XMUL(H, om.ambda[KE]);
    double F1, F2, F3, F4, X1, X2, X3, X4, Y1, Y2, Y3, Y4, Z1, Z2, Z3, Z4;
    vsd(P, JJ, XGI, YGI, XSUB(ZP1, HA), F1, X1, Y1, Z1);
    vsd(P, JJ, XGI, YGI, XSUB(ZP2, HA), F2, X2, Y2, Z2);
    vsd(P, JJ, XGI, YGI, XADD(ZP3, HA), F3, X3, Y3, Z3);
    vsd(P, JJ, XGI, YGI, XADD(ZP4, HA), F4, X4, Y4, Z4);
    const double ar = om.ar[KE];
    w.FS1 += (F1 + F2 + F3 + F4) * ar;
    w.VSX1 += (X1 + X2 + X3 + X4) * ar;
    w.VSY1 += (Y1 + Y2 + Y3 + Y4) * ar;
    w.VSZ1 += (-Z1 + Z2 + Z3 - Z4) * ar;
  }
}

// one tabulated image of VNSFD (blocks 0001-0012 and 601B)
struct FdImage {
  double PD1Z, PD2Z, VZ2, PD1X, VR2, PSR;
};

__device__ __forceinline__ void fd_image(const GreenCtx& g, double AM0, double AKR, double RRR, double ZZZ,
                                         const Lagrange& LX, bool tab, double PSK, double SCK, double SCDS,
                                         double SSDS, FdImage& m, bool& bad) {
  const double PI = 3.141592653589793, EPS = 0.0001;
  const double AKZ = XMUL(AM0, ZZZ);
  const double DD = XSQRT(XADD(XMUL(RRR, RRR), XMUL(ZZZ, ZZZ)));
  double PSURR = 0.;
  m.PSR = 0.;
  if (DD > EPS) {
    double RRv = AM0 * DD;
    m.PSR = PI / RRv;
    PSURR = PI / (RRv * RRv * RRv);
  }
  if (AKZ > -1.5E-6) {
    bad = true;
    m = FdImage{0, 0, 0, 0, 0, 0};
    return;
  }
  if (AKZ > -16.) {
    double PD1X, PD2X;
    if (tab) {
      Lagrange L = LX;
      lagrange_z(g, AKZ, L);
      double4 t = interp4(g, L);
      PD1X = t.x; m.PD1Z = t.y; PD2X = t.z; m.PD2Z = t.w;
    } else {
      double EPZ = exp(AKZ);
      m.PD1Z = PSURR * AKZ - PSK * EPZ;
      m.PD2Z = EPZ * SCK;
      PD1X = -PSURR * AKR - EPZ * SCDS;
      PD2X = EPZ * SSDS;
    }
    m.VZ2 = m.PD2Z;
    m.PD1X = PD1X;
    m.VR2 = -PD2X;
  } else {
    m.PD1Z = PSURR * AKZ;
    m.PD2Z = 0.;
    m.VZ2 = 0.;
    m.PD1X = -PSURR * AKR;
    m.VR2 = 0.;
  }
}

// --- VNSFD for one reflection BX ------------------------------------------
__device__ __forceinline__ void wave_fd_jj(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI,
                                           double ZMIII, int BX, const PanelRec& P, WaveJJ& w) {
  const double PI = 3.141592653589793, PI4 = 0.7853981633974483, DPI = 2. * PI, EPS = 0.0001;
  const double QPI = 4. * PI;
  const double AM0 = om.k0, H = om.h;
  const double YMJJJ = P.yg * BX;
  const double COF1 = om.coe3 * P.aire, COF2 = om.coe4 * P.aire;
  const double COF3 = AM0 * COF1, COF4 = AM0 * COF2;
  const double dx = XSUB(XGI, P.xg), dy = XSUB(YGI, YMJJJ);
  const double RRR = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
  const double AKR = XMUL(AM0, RRR);
  const double H2 = XMUL(2., H), H4 = XMUL(4., H);
  const double Z1 = XADD(ZMIII, P.zg);
  const double Z2 = XSUB(XSUB(P.zg, ZMIII), H2);
  const double Z3 = XSUB(XSUB(ZMIII, P.zg), H2);
  const double Z4 = XSUB(XSUB(-P.zg, ZMIII), H4);
  const bool tab = AKR < 99.7;
  Lagrange LX{};
  double PSK = 0., SCK = 0., SCDS = 0., SSDS = 0.;
  const double AKZ1 = XMUL(AM0, Z1);
  if (AKZ1 > -16. && AKZ1 <= -1.5E-6) {
    if (tab) {
      lagrange_x(g, AKR, LX);
    } else {
      double SQ = sqrt(DPI / AKR), SIK, CSK;
      sincos(AKR - PI4, &SIK, &CSK);
      PSK = PI * SQ * SIK;
      SCK = SQ * CSK;
      double DSK = 0.5 / AKR;
      SCDS = PI * SQ * (CSK - DSK * SIK);
      SSDS = SQ * (SIK + DSK * CSK);
    }
  }
  bool bad = false;
  FdImage m1, m2, m3, m4;
  fd_image(g, AM0, AKR, RRR, Z1, LX, tab, PSK, SCK, SCDS, SSDS, m1, bad);
  fd_image(g, AM0, AKR, RRR, Z2, LX, tab, PSK, SCK, SCDS, SSDS, m2, bad);
  fd_image(g, AM0, AKR, RRR, Z3, LX, tab, PSK, SCK, SCDS, SSDS, m3, bad);
  fd_image(g, AM0, AKR, RRR, Z4, LX, tab, PSK, SCK, SCDS, SSDS, m4, bad);
  if (bad) {
    set_status(g.status, ST_AKZ_UNDEFINED);
    w = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
    return;
  }
  w.FS1 = COF1 * ((m1.PD1Z + m2.PD1Z + m3.PD1Z + m4.PD1Z) - m1.PSR - m2.PSR - m3.PSR - m4.PSR);
  w.FS2 = COF2 * (m1.PD2Z + m2.PD2Z + m3.PD2Z + m4.PD2Z);
  if (RRR > EPS) {
    const double C1V3 = -COF3 * (m1.PD1X + m2.PD1X + m3.PD1X + m4.PD1X);
    const double C2V3 = COF4 * (m1.VR2 + m2.VR2 + m3.VR2 + m4.VR2);
    const double iR = 1. / RRR;
    const double CVX = dx * iR, CVY = dy * iR;
    w.VSX1 = C1V3 * CVX;
    w.VSX2 = C2V3 * CVX;
    w.VSY1 = C1V3 * CVY;
    w.VSY2 = C2V3 * CVY;
  } else {
    w.VSX1 = w.VSX2 = w.VSY1 = w.VSY2 = 0.;
  }
  w.VSZ1 = COF3 * (m1.PD1Z - m2.PD1Z + m3.PD1Z - m4.PD1Z);
  w.VSZ2 = COF4 * (m1.VZ2 - m2.VZ2 + m3.VZ2 - m4.VZ2);
  // the exponential images (:635-706) are added by fd_images_kernel
}

// --- one pair, both symmetry classes --------------------------------------
template <bool FD>
__device__ __forceinline__ void pair_green(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI, double ZGI,
                                           double XNI, double YNI, double ZNI, bool self, const PanelRec& P,
                                           PairOut& out) {
  RankineOut r;
  rankine<FD>(g, FD ? XMUL(2., om.h) : 0., XGI, YGI, ZGI, self, P, r);
  const int NJJ = g.nsymy + 1;
  double ZMIII = ZGI;
  if (ZGI > g.zer) ZMIII = FD ? XMUL(20., g.zer) : g.zer;
  const bool tabulated = (ZGI < g.zer) && (P.zg < g.zer);
  WaveJJ w[2];
#pragma unroll
  for (int JJ = 1; JJ <= 2; ++JJ) {
    if (JJ > NJJ) break;
    const int BX = (JJ == 1) ? 1 : -1;
    if (tabulated) {
      if (FD) wave_fd_jj(g, om, XGI, YGI, ZMIII, BX, P, w[JJ - 1]);
      else wave_infd_jj(g, om, XGI, YGI, ZMIII, BX, P, w[JJ - 1]);
    } else {
      if (FD) wave_fd_fs(om, XGI, YGI, ZMIII, JJ, P, w[JJ - 1]);
      else wave_infd_fs(om, XGI, YGI, ZMIII, BX, P, w[JJ - 1]);
    }
  }
  double SP1, SM1, SP2, SM2, VXP1, VXM1, VYP1, VYM1, VZP1, VZM1, VXP2, VXM2, VYP2, VYM2, VZP2, VZM2;
  if (!FD) {
    // VNSINFD combination (:456-500)
    const double DPI = 2. * 3.141592653589793, DPI2 = 2. * 3.141592653589793 * 3.141592653589793;
    const double AKAIR = om.k0 * P.aire;
    const double ADPI2 = AKAIR / DPI2, ADPI = AKAIR / DPI;
    const double AKDPI2 = ADPI2 * om.k0, AKDPI = ADPI * om.k0;
    if (NJJ == 2) {
      SM1 = r.FSM - (w[0].FS1 - w[1].FS1) * ADPI2;
      SP1 = r.FSP - (w[0].FS1 + w[1].FS1) * ADPI2;
      SM2 = -(w[0].FS2 - w[1].FS2) * ADPI;
      SP2 = -(w[0].FS2 + w[1].FS2) * ADPI;
      VXP1 = r.VSXP - (w[0].VSX1 + w[1].VSX1) * AKDPI2;
      VXM1 = r.VSXM - (w[0].VSX1 - w[1].VSX1) * AKDPI2;
      VYP1 = r.VSYP - (w[0].VSY1 + w[1].VSY1) * AKDPI2;
      VYM1 = r.VSYM - (w[0].VSY1 - w[1].VSY1) * AKDPI2;
      VZP1 = r.VSZP - (w[0].VSZ1 + w[1].VSZ1) * AKDPI2;
      VZM1 = r.VSZM - (w[0].VSZ1 - w[1].VSZ1) * AKDPI2;
      VXP2 = -(w[0].VSX2 + w[1].VSX2) * AKDPI;
      VXM2 = -(w[0].VSX2 - w[1].VSX2) * AKDPI;
      VYP2 = -(w[0].VSY2 + w[1].VSY2) * AKDPI;
      VYM2 = -(w[0].VSY2 - w[1].VSY2) * AKDPI;
      VZP2 = -(w[0].VSZ2 + w[1].VSZ2) * AKDPI;
      VZM2 = -(w[0].VSZ2 - w[1].VSZ2) * AKDPI;
    } else {
      SP1 = SM1 = r.FSP - w[0].FS1 * ADPI2;
      SP2 = SM2 = -w[0].FS2 * ADPI;
      VXP1 = VXM1 = r.VSXP - w[0].VSX1 * AKDPI2;
      VYP1 = VYM1 = r.VSYP - w[0].VSY1 * AKDPI2;
      VZP1 = VZM1 = r.VSZP - w[0].VSZ1 * AKDPI2;
      VXP2 = VXM2 = -w[0].VSX2 * AKDPI;
      VYP2 = VYM2 = -w[0].VSY2 * AKDPI;
      VZP2 = VZM2 = -w[0].VSZ2 * AKDPI;
    }
  } else {
    // VNSFD combination (:830-865)
    if (NJJ == 2) {
      SM1 = r.FSM + w[0].FS1 - w[1].FS1;
      SP1 = r.FSP + w[0].FS1 + w[1].FS1;
      SM2 = w[0].FS2 - w[1].FS2;
      SP2 = w[0].FS2 + w[1].FS2;
      VXP1 = r.VSXP + w[0].VSX1 + w[1].VSX1;
      VXM1 = r.VSXM + w[0].VSX1 - w[1].VSX1;
      VYP1 = r.VSYP + w[0].VSY1 + w[1].VSY1;
      VYM1 = r.VSYM + w[0].VSY1 - w[1].VSY1;
      VZP1 = r.VSZP + w[0].VSZ1 + w[1].VSZ1;
      VZM1 = r.VSZM + w[0].VSZ1 - w[1].VSZ1;
      VXP2 = w[0].VSX2 + w[1].VSX2;
      VXM2 = w[0].VSX2 - w[1].VSX2;
      VYP2 = w[0].VSY2 + w[1].VSY2;
      VYM2 = w[0].VSY2 - w[1].VSY2;
      VZP2 = w[0].VSZ2 + w[1].VSZ2;
      VZM2 = w[0].VSZ2 - w[1].VSZ2;
    } else {
      SP1 = SM1 = r.FSP + w[0].FS1;
      SP2 = SM2 = w[0].FS2;
      VXP1 = VXM1 = r.VSXP + w[0].VSX1;
      VYP1 = VYM1 = r.VSYP + w[0].VSY1;
      VZP1 = VZM1 = r.VSZP + w[0].VSZ1;
      VXP2 = VXM2 = w[0].VSX2;
      VYP2 = VYM2 = w[0].VSY2;
      VZP2 = VZM2 = w[0].VSZ2;
    }
  }
  out.dp_re = VXP1 * XNI + VYP1 * YNI + VZP1 * ZNI;
  out.dp_im = VXP2 * XNI + VYP2 * YNI + VZP2 * ZNI;
  out.dm_re = VXM1 * XNI + VYM1 * YNI + VZM1 * ZNI;
  out.dm_im = VXM2 * XNI + VYM2 * YNI + VZM2 * ZNI;
  out.sp_re = SP1;
  out.sp_im = SP2;
  out.sm_re = SM1;
  out.sm_im = SM2;
}

}  // namespace nb200
