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
  const double4* xlag;              // 3-node Lagrange stencils of XR, two double4 per centre node K
  const double4* zlag;              // same for XZ
  const StencilThresholds* thr;
  double zer;                       // ZER (PREPARE_MESH.f90:58-69)
  int nsymy;
  int* status;                      // device status word (first error wins)
};

struct PairOut {
  double dp_re, dp_im, dm_re, dm_im;  // D+, D-
  double sp_re, sp_im, sm_re, sm_im;  // S+, S-
};

NB_HD __forceinline__ void set_status(int* st, int code) {
#ifdef __CUDA_ARCH__
  atomicCAS(st, 0, code);
#else
  if (*st == 0) *st = code;
#endif
}

// --- GG(Z,CEX): ELEMENTARY_FNS.f90:31-81 ----------------------------------
NB_HD __noinline__ cplx GG(cplx Z, cplx CEX) {
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

// integer part of a monotone log10 expression, made exact by thresholds: the
// estimate k may be off by up to four (it comes from an FP32 log10, within one
// of the exact value), the thresholds settle it
NB_HD __forceinline__ int stencil_adjust(double x, const double* thr, int k) {
  k = max(0, min(k, 47));
#pragma unroll 1
  for (int it = 0; it < 4 && k < 47 && x >= NB_LDG(thr + k + 1); ++it) ++k;
#pragma unroll 1
  for (int it = 0; it < 4 && k > 0 && x < NB_LDG(thr + k); ++it) --k;
  return k;
}

// KJ of COMPUTE_GREEN_INFD.f90:292-298 (AKZ in (-16, -1.5e-6])
NB_HD __forceinline__ int stencil_kj(double AKZ, const StencilThresholds* T) {
  double x = -AKZ;
  int k;
  const float lx = log10f((float)x);
  if (AKZ < -1.E-2) k = stencil_adjust(x, T->kj8, (int)(8.f * (lx + 4.5f)));
  else k = stencil_adjust(x, T->kj5, (int)(5.f * (lx + 6.f)));
  k = max(k, 2);
  return min(k, 45);
}

// KI of COMPUTE_GREEN_INFD.f90:299-305
NB_HD __forceinline__ int stencil_ki(double AKR, const StencilThresholds* T) {
  int k;
  if (AKR < 1.) {
    double y = XADD(AKR, 1.E-20);
    k = stencil_adjust(y, T->ki5, (int)(5.f * (log10f((float)y) + 6.f) + 1.f));
  } else {
    k = (int)XADD(XMUL(3., AKR), 28.);
  }
  k = max(k, 2);
  return min(k, 327);
}

// Three-node Lagrange stencil around node K of a table axis: the reference
// evaluates PL2(U1,U2,U3,XU) = (XU-U1)(XU-U2)/((U3-U1)(U3-U2)) on the nodes
// K-1, K, K+1 (COMPUTE_GREEN_INFD.f90:306-311, :641-645). The nodes and the
// reciprocals of the three denominators are tabulated per K (two double4:
// {a, b, c, 1/((a-b)(a-c))}, {1/((b-c)(b-a)), 1/((c-a)(c-b)), 0, 0}), so a
// coefficient is two products instead of a division.
struct Stencil {
  int K;
  double L1, L2, L3;
};

NB_HD __forceinline__ double4 ldg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = NB_LDG(q), b = NB_LDG(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

NB_HD __forceinline__ void stencil_coeffs(const double4* lag, int K, double u, Stencil& s) {
  const double4 p = ldg4(lag + 2 * K), q = ldg4(lag + 2 * K + 1);
  s.K = K;
  s.L1 = ((u - p.y) * (u - p.z)) * p.w;
  s.L2 = ((u - p.z) * (u - p.x)) * q.x;
  s.L3 = ((u - p.x) * (u - p.y)) * q.y;
}

NB_HD __forceinline__ void stencil_x(const GreenCtx& g, double AKR, Stencil& s) {
  stencil_coeffs(g.xlag, stencil_ki(AKR, g.thr), AKR, s);
}
NB_HD __forceinline__ void stencil_z(const GreenCtx& g, double AKZ, Stencil& s) {
  stencil_coeffs(g.zlag, stencil_kj(AKZ, g.thr), AKZ, s);
}

// 3x3 Lagrange interpolation of the four tables (:306-319, :345-352)
NB_HD __forceinline__ double4 interp4(const GreenCtx& g, const Stencil& sx, const Stencil& sz) {
  double4 r = make_double4(0., 0., 0., 0.);
  const double zl[3] = {sz.L1, sz.L2, sz.L3};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const double4* row = g.apd + (sx.K - 2) + TAB_IR * (sz.K - 2 + b);
    double4 t1 = ldg4(row), t2 = ldg4(row + 1), t3 = ldg4(row + 2);
    double4 F;
    F.x = sx.L1 * t1.x + sx.L2 * t2.x + sx.L3 * t3.x;
    F.y = sx.L1 * t1.y + sx.L2 * t2.y + sx.L3 * t3.y;
    F.z = sx.L1 * t1.z + sx.L2 * t2.z + sx.L3 * t3.z;
    F.w = sx.L1 * t1.w + sx.L2 * t2.w + sx.L3 * t3.w;
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
NB_HD __noinline__ void rankine_near(double XOI, double YOI, double ZOI, const PanelRec& P, int MY, int MZ,
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

// Images JJ = 1..4 (direct, sea-bottom / free-surface image, and their
// y-mirrors) are combined into the two symmetry classes as they are computed:
// class + takes (1, -MK, -MK, 1), class - takes (1, -MK, MK, -1) of the four
// (VAVINFD/VAVFD combination, COMPUTE_GREEN_INFD.f90:176-216).
template <bool FD>
NB_HD __forceinline__ void rankine(const GreenCtx& g, double DH, double XGI, double YGI, double ZGI, bool self,
                                        const PanelRec& P, RankineOut& o, bool clip = true) {
  const double QPI = 4. * 3.141592653589793;
  const double DPI = 2. * 3.141592653589793;
  const int NJJ = 2 * (g.nsymy + 1);
  const double MK = FD ? -1. : 1.;
  double XOI = XGI, YOI = YGI, ZOI = ZGI;
  if (clip && ZGI > g.zer) ZOI = FD ? XMUL(20., g.zer) : g.zer;
  const double lim7 = XMUL(7., P.tdis);
  o = RankineOut{0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
  for (int JJ = 1; JJ <= NJJ; ++JJ) {
    const int MJJ = (JJ & 1) ? 1 : -1;
    const int MY = (JJ >= 3) ? -1 : 1;
    const int MZ = (JJ == 2 || JJ == 3) ? -1 : 1;
    const double DHMH = (JJ == 2 || JJ == 3) ? DH : 0.;
    const double XOJ = P.xg, YOJ = P.yg * MY, ZOJ = XSUB(P.zg * MZ, DHMH);
    const double dx = XSUB(XOI, XOJ), dy = XSUB(YOI, YOJ), dz = XSUB(ZOI, ZOJ);
    const double RO = XSQRT(XADD(XADD(XMUL(dx, dx), XMUL(dy, dy)), XMUL(dz, dz)));
    double a, vx, vy, vz;
    if (RO > lim7) {
      const double iRO = 1. / RO;
      a = P.aire * iRO;
      const double ASRO = a * iRO * iRO;
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
    const double cp = (JJ == 1 || JJ == 4) ? 1. : -MK;
    const double cm = (JJ == 1) ? 1. : (JJ == 2) ? -MK : (JJ == 3) ? MK : -1.;
    o.FSP += cp * a; o.VSXP += cp * vx; o.VSYP += cp * vy; o.VSZP += cp * vz;
    o.FSM += cm * a; o.VSXM += cm * vx; o.VSYM += cm * vy; o.VSZM += cm * vz;
  }
  const double iq = -1. / QPI;
  if (g.nsymy == 1) {
    o.FSP *= iq; o.VSXP *= iq; o.VSYP *= iq; o.VSZP *= iq;
    o.FSM *= iq; o.VSXM *= iq; o.VSYM *= iq; o.VSZM *= iq;
  } else {
    o.FSP *= iq; o.VSXP *= iq; o.VSYP *= iq; o.VSZP *= iq;
    o.FSM = o.FSP; o.VSXM = o.VSXP; o.VSYM = o.VSYP; o.VSZM = o.VSZP;
  }
}

// per-reflection wave contributions (FS1..VSZ2 of one JJ)
struct WaveJJ {
  double FS1, FS2, VSX1, VSY1, VSZ1, VSX2, VSY2, VSZ2;
};

// --- VNSINFD free-surface-panel branch (COMPUTE_GREEN_INFD.f90:385-453) ---
NB_HD __noinline__ void wave_infd_fs(const OmegaParams& om, double XGI, double YGI, double ZMIII, int BX,
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

// --- VNSINFD tabulated branch, both reflections (:271-382) ----------------
// AKZ depends on the depths only, so its stencil is shared by BX = +1 and -1.
NB_HD __forceinline__ void wave_infd_pair(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI,
                                               double ZMIII, const PanelRec& P, int NJJ, WaveJJ* w) {
  const double PI = 3.141592653589793, PI4 = 0.7853981633974483, DPI = 2. * PI, EPS = 0.0001;
  const double AK0 = om.k0;
  const double ZZZ = XADD(ZMIII, P.zg);
  const double AKZ = XMUL(AK0, ZZZ);
  if (AKZ > -1.5E-6) {
    set_status(g.status, ST_AKZ_UNDEFINED);
    w[0] = w[1] = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
    return;
  }
  Stencil sz;
  bool have_sz = false;
#pragma unroll 1
  for (int b = 0; b < NJJ; ++b) {
    const double YMJJJ = b ? -P.yg : P.yg;
    const double dx = XSUB(XGI, P.xg), dy = XSUB(YGI, YMJJJ);
    const double RRR = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
    const double AKR = XMUL(AK0, RRR);
    const double DD = XSQRT(XADD(XMUL(RRR, RRR), XMUL(ZZZ, ZZZ)));
    double PSURR = 0.;
    if (DD > EPS) {
      const double it = 1. / (AK0 * DD);
      PSURR = PI * it * it * it;
    }
    double PD1Z, PD2Z, VZ1, VZ2, PD1X = 0., PD2X = 0., VR1 = 0., VR2 = 0.;
    if (AKZ > -16.) {
      if (AKR < 99.7) {
        if (!have_sz) {
          stencil_z(g, AKZ, sz);
          have_sz = true;
        }
        Stencil sx;
        stencil_x(g, AKR, sx);
        const double4 t = interp4(g, sx, sz);
        PD1X = t.x; PD1Z = t.y; PD2X = t.z; PD2Z = t.w;
      } else {
        const double EPZ = exp(AKZ);
        const double SQ = sqrt(DPI / AKR);
        double SIK, CSK;
        sincos(AKR - PI4, &SIK, &CSK);
        PD1Z = PSURR * AKZ - PI * EPZ * SQ * SIK;
        PD2Z = EPZ * SQ * CSK;
        const double DSK = 0.5 / AKR;
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
    WaveJJ& o = w[b];
    o.FS1 = PD1Z;
    o.FS2 = PD2Z;
    if (RRR > EPS) {
      const double iR = 1. / RRR;
      const double CVX = dx * iR, CVY = dy * iR;
      o.VSX1 = VR1 * CVX;
      o.VSX2 = VR2 * CVX;
      o.VSY1 = VR1 * CVY;
      o.VSY2 = VR2 * CVY;
    } else {
      o.VSX1 = o.VSX2 = o.VSY1 = o.VSY2 = 0.;
    }
    o.VSZ1 = VZ1;
    o.VSZ2 = VZ2;
  }
}

// --- VSD: exact Rankine panel integral used by the FD free-surface branch --
// (COMPUTE_GREEN_FD.f90:1514-1609)
NB_HD __noinline__ void vsd(const PanelRec& P, int JJ, double XGI, double YGI, double ZIG, double& FS, double& VX,
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
NB_HD __noinline__ void wave_fd_fs(const OmegaParams& om, double XGI, double YGI, double ZMIII, int JJ,
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

NB_HD __forceinline__ void fd_image(const GreenCtx& g, double AM0, double AKR, double RRR, double ZZZ, double AKZ,
                                         const Stencil& sx, const Stencil& sz, bool tab, double PSK, double SCK,
                                         double SCDS, double SSDS, FdImage& m) {
  const double PI = 3.141592653589793, EPS = 0.0001;
  const double DD = XSQRT(XADD(XMUL(RRR, RRR), XMUL(ZZZ, ZZZ)));
  double PSURR = 0.;
  m.PSR = 0.;
  if (DD > EPS) {
    const double it = 1. / (AM0 * DD);
    m.PSR = PI * it;
    PSURR = m.PSR * it * it;
  }
  if (AKZ > -16.) {
    double PD1X, PD2X;
    if (tab) {
      const double4 t = interp4(g, sx, sz);
      PD1X = t.x; m.PD1Z = t.y; PD2X = t.z; m.PD2Z = t.w;
    } else {
      const double EPZ = exp(AKZ);
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

// --- VNSFD tabulated branch, both reflections ------------------------------
// The four image depths Z1..Z4 (and their AKZ stencils) depend on the depths
// only and are shared by BX = +1 and -1. |Z1| is the smallest of the four,
// so AKZ1 <= -16 puts every image in the far branch.
NB_HD __forceinline__ void wave_fd_pair(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI,
                                             double ZMIII, const PanelRec& P, int NJJ, WaveJJ* w) {
  const double PI = 3.141592653589793, PI4 = 0.7853981633974483, DPI = 2. * PI, EPS = 0.0001;
  const double AM0 = om.k0, H = om.h;
  const double COF1 = om.coe3 * P.aire, COF2 = om.coe4 * P.aire;
  const double COF3 = AM0 * COF1, COF4 = AM0 * COF2;
  const double H2 = XMUL(2., H), H4 = XMUL(4., H);
  double Z[4], AKZ[4];
  Z[0] = XADD(ZMIII, P.zg);
  Z[1] = XSUB(XSUB(P.zg, ZMIII), H2);
  Z[2] = XSUB(XSUB(ZMIII, P.zg), H2);
  Z[3] = XSUB(XSUB(-P.zg, ZMIII), H4);
  bool bad = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    AKZ[k] = XMUL(AM0, Z[k]);
    bad |= AKZ[k] > -1.5E-6;
  }
  if (bad) {
    set_status(g.status, ST_AKZ_UNDEFINED);
    w[0] = w[1] = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
    return;
  }
  const bool near = AKZ[0] > -16.;
  Stencil sz[4];
  bool have_sz = false;
#pragma unroll 1
  for (int b = 0; b < NJJ; ++b) {
    const double YMJJJ = b ? -P.yg : P.yg;
    const double dx = XSUB(XGI, P.xg), dy = XSUB(YGI, YMJJJ);
    const double RRR = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
    const double AKR = XMUL(AM0, RRR);
    const bool tab = AKR < 99.7;
    Stencil sx{2, 0., 0., 0.};
    double PSK = 0., SCK = 0., SCDS = 0., SSDS = 0.;
    if (near) {
      if (tab) {
        stencil_x(g, AKR, sx);
        if (!have_sz) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (AKZ[k] > -16.) stencil_z(g, AKZ[k], sz[k]);
          have_sz = true;
        }
      } else {
        const double SQ = sqrt(DPI / AKR);
        double SIK, CSK;
        sincos(AKR - PI4, &SIK, &CSK);
        PSK = PI * SQ * SIK;
        SCK = SQ * CSK;
        const double DSK = 0.5 / AKR;
        SCDS = PI * SQ * (CSK - DSK * SIK);
        SSDS = SQ * (SIK + DSK * CSK);
      }
    }
    FdImage m[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) fd_image(g, AM0, AKR, RRR, Z[k], AKZ[k], sx, sz[k], tab, PSK, SCK, SCDS, SSDS, m[k]);
    WaveJJ& o = w[b];
    o.FS1 = COF1 * ((m[0].PD1Z + m[1].PD1Z + m[2].PD1Z + m[3].PD1Z) - m[0].PSR - m[1].PSR - m[2].PSR - m[3].PSR);
    o.FS2 = COF2 * (m[0].PD2Z + m[1].PD2Z + m[2].PD2Z + m[3].PD2Z);
    if (RRR > EPS) {
      const double C1V3 = -COF3 * (m[0].PD1X + m[1].PD1X + m[2].PD1X + m[3].PD1X);
      const double C2V3 = COF4 * (m[0].VR2 + m[1].VR2 + m[2].VR2 + m[3].VR2);
      const double iR = 1. / RRR;
      const double CVX = dx * iR, CVY = dy * iR;
      o.VSX1 = C1V3 * CVX;
      o.VSX2 = C2V3 * CVX;
      o.VSY1 = C1V3 * CVY;
      o.VSY2 = C2V3 * CVY;
    } else {
      o.VSX1 = o.VSX2 = o.VSY1 = o.VSY2 = 0.;
    }
    o.VSZ1 = COF3 * (m[0].PD1Z - m[1].PD1Z + m[2].PD1Z - m[3].PD1Z);
    o.VSZ2 = COF4 * (m[0].VZ2 - m[1].VZ2 + m[2].VZ2 - m[3].VZ2);
  }
}

// --- VNSFD tabulated branch for both orders of a pair ------------------------
// With both panels submerged the four image depths of (I, J) are
//   Z1 = ZI + ZJ, Z2 = (ZJ - ZI) - 2h, Z3 = (ZI - ZJ) - 2h, Z4 = (-ZJ - ZI) - 4h
// and those of (J, I) are the same numbers with Z2 and Z3 exchanged; the
// horizontal distances agree as well. So one set of table interpolations
// serves both orders: the sums over the images are shared, and the z
// gradient PD1Z1 - PD1Z2 + PD1Z3 - PD1Z4 of (I, J) is PD1Z1 + PD1Z2 - PD1Z3 -
// PD1Z4 for (J, I). The x and the direct-reflection y distances change sign
// with the order, the mirror's y distance does not. Each reflection is added
// to the symmetry classes (+ both, - with the mirror subtracted) of the two
// orders as it is computed. Returns false (and leaves the outputs) when an
// image depth is too shallow for the tables (AKZ > -1.5e-6).
NB_HD __forceinline__ void wave_sym_add(const OmegaParams& om, double aire, double XN, double YN, double ZN,
                                             double sgn, double F1, double F2, double X1, double X2, double ZA1,
                                             double ZA2, double CVX, double CVY, PairOut& o) {
  const double COF1 = om.coe3 * aire, COF2 = om.coe4 * aire;
  const double COF3 = om.k0 * COF1, COF4 = om.k0 * COF2;
  const double FS1 = COF1 * F1, FS2 = COF2 * F2;
  const double C1V3 = -COF3 * X1, C2V3 = COF4 * X2;
  const double D1 = (C1V3 * CVX) * XN + (C1V3 * CVY) * YN + (COF3 * ZA1) * ZN;
  const double D2 = (C2V3 * CVX) * XN + (C2V3 * CVY) * YN + (COF4 * ZA2) * ZN;
  o.sp_re += FS1;
  o.sm_re += sgn * FS1;
  o.sp_im += FS2;
  o.sm_im += sgn * FS2;
  o.dp_re += D1;
  o.dm_re += sgn * D1;
  o.dp_im += D2;
  o.dm_im += sgn * D2;
}

NB_HD __forceinline__ bool wave_fd_sym(const GreenCtx& g, const OmegaParams& om, const PanelRec& PI,
                                            const PanelRec& PJ, int NJJ, bool both, PairOut& oij, PairOut& oji) {
  const double PI_ = 3.141592653589793, PI4 = 0.7853981633974483, DPI = 2. * PI_, EPS = 0.0001;
  const double AM0 = om.k0, H = om.h;
  const double H2 = XMUL(2., H), H4 = XMUL(4., H);
  double Z[4], AKZ[4];
  Z[0] = XADD(PI.zg, PJ.zg);
  Z[1] = XSUB(XSUB(PJ.zg, PI.zg), H2);
  Z[2] = XSUB(XSUB(PI.zg, PJ.zg), H2);
  Z[3] = XSUB(XSUB(-PJ.zg, PI.zg), H4);
  bool bad = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    AKZ[k] = XMUL(AM0, Z[k]);
    bad |= AKZ[k] > -1.5E-6;
  }
  if (bad) return false;
  oij = PairOut{0, 0, 0, 0, 0, 0, 0, 0};
  oji = oij;
  const bool near = AKZ[0] > -16.;
  Stencil sz[4];
  bool have_sz = false;
#pragma unroll 1
  for (int b = 0; b < NJJ; ++b) {
    const double YMJJJ = b ? -PJ.yg : PJ.yg;
    const double dx = XSUB(PI.xg, PJ.xg), dy = XSUB(PI.yg, YMJJJ);
    const double RRR = XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy)));
    const double AKR = XMUL(AM0, RRR);
    const bool tab = AKR < 99.7;
    Stencil sx{2, 0., 0., 0.};
    double PSK = 0., SCK = 0., SCDS = 0., SSDS = 0.;
    if (near) {
      if (tab) {
        stencil_x(g, AKR, sx);
        if (!have_sz) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (AKZ[k] > -16.) stencil_z(g, AKZ[k], sz[k]);
          have_sz = true;
        }
      } else {
        const double SQ = sqrt(DPI / AKR);
        double SIK, CSK;
        sincos(AKR - PI4, &SIK, &CSK);
        PSK = PI_ * SQ * SIK;
        SCK = SQ * CSK;
        const double DSK = 0.5 / AKR;
        SCDS = PI_ * SQ * (CSK - DSK * SIK);
        SSDS = SQ * (SIK + DSK * CSK);
      }
    }
    // image by image into running sums: z gradients with the signs of
    // (I, J) (+ - + -) and of (J, I) (+ + - -)
    double s1z = 0., spsr = 0., s2z = 0., s1x = 0., s2r = 0., zp1 = 0., zq1 = 0., zp2 = 0., zq2 = 0.;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      FdImage m;
      fd_image(g, AM0, AKR, RRR, Z[k], AKZ[k], sx, sz[k], tab, PSK, SCK, SCDS, SSDS, m);
      const double sp = (k & 1) ? -1. : 1., sq = (k < 2) ? 1. : -1.;
      s1z += m.PD1Z;
      spsr += m.PSR;
      s2z += m.PD2Z;
      s1x += m.PD1X;
      s2r += m.VR2;
      zp1 += sp * m.PD1Z;
      zq1 += sq * m.PD1Z;
      zp2 += sp * m.VZ2;
      zq2 += sq * m.VZ2;
    }
    const double F1 = s1z - spsr;
    const double iR = RRR > EPS ? 1. / RRR : 0.;
    const double sgn = b ? -1. : 1.;
    wave_sym_add(om, PJ.aire, PI.xn, PI.yn, PI.zn, sgn, F1, s2z, s1x, s2r, zp1, zp2, dx * iR, dy * iR, oij);
    if (both)
      wave_sym_add(om, PI.aire, PJ.xn, PJ.yn, PJ.zn, sgn, F1, s2z, s1x, s2r, zq1, zq2, -dx * iR,
                   (b ? dy : -dy) * iR, oji);
  }
  if (NJJ == 1) {   // one class: the minus entries equal the plus ones
    oij.sm_re = oij.sp_re; oij.sm_im = oij.sp_im; oij.dm_re = oij.dp_re; oij.dm_im = oij.dp_im;
    oji.sm_re = oji.sp_re; oji.sm_im = oji.sp_im; oji.dm_re = oji.dp_re; oji.dm_im = oji.dp_im;
  }
  return true;
}

// --- VNSFD exponential images (COMPUTE_GREEN_FD.f90:635-706) ----------------
//   sum_KE AR(KE) (-A_J/8pi) sum_4 1/rho  and their gradients, per reflection.
// The reference adds them to FS1, VSX1, VSY1, VSZ1 of each reflection, and
// those enter SP1/SM1 and the real parts of D+/- linearly (:830-865). Image
// depths are shared by both reflections; RO > EPS is decided exactly on RO^2
// against a precomputed threshold.
//
// The four image depths of collocation I and panel J are
//   z0 = ZI - 2h + h l - ZJ,  z1 = -ZI - h l - ZJ,  z2 = -ZI - 4h + h l - ZJ,
//   z3 = ZI + 2h - h l - ZJ,
// and exchanging I and J maps z0 -> -z3, z3 -> -z0 and keeps z1, z2; the
// horizontal distance of both reflections is unchanged. So one evaluation of
// the 4 (NEXP+1) reciprocal distances of an unordered pair serves both
// ordered pairs. Per reflection b it returns, without the panel factor
// ACT = -A/8pi,
//   fs = sum AR sum_k 1/rho_k,        sa = sum AR sum_k 1/rho_k^3,
//   m1 = sum AR (z0 a0 - z1 a1 - z2 a2 + z3 a3),
//   m2 = sum AR (z0 a0 + z1 a1 + z2 a2 + z3 a3),   a_k = 1/rho_k^3,
// from which the pair (I, J) takes fs, -dx sa, -dy sa, -m1 (times ACT_J) and
// the pair (J, I) takes fs, dx sa, -dy' sa, +m2 (times ACT_I), dy' being the
// y distance of (J, I) (-dy for the direct reflection, dy for the mirror).
struct ImageSums {
  double fs[2], sa[2], m1[2], m2[2], dx[2], dy[2];
};

NB_HD __forceinline__ void fd_image_sums(const GreenCtx& g, double H, const double* ambda, const double* ar,
                                              int nexp1, double XI, double YI, double ZI, double XJ, double YJ,
                                              double ZJ, int NJJ, ImageSums& o) {
  const double H2 = XMUL(2., H), H4 = XMUL(4., H);
  const double T2 = g.ro_eps2;
  double r2[2];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    o.fs[b] = o.sa[b] = o.m1[b] = o.m2[b] = 0.;
    o.dx[b] = XSUB(XI, XJ);
    o.dy[b] = XSUB(YI, YJ * (b ? -1. : 1.));
    const double R = XSQRT(XADD(XMUL(o.dx[b], o.dx[b]), XMUL(o.dy[b], o.dy[b])));
    r2[b] = XMUL(R, R);
  }
#pragma unroll 1
  for (int KE = 1; KE <= nexp1; ++KE) {
    const double A = ar[KE];
    const double HA = XMUL(H, ambda[KE]);
    double zp[4], z2[4];
    zp[0] = XSUB(XADD(XSUB(ZI, H2), HA), ZJ);
    zp[1] = XSUB(XSUB(-ZI, HA), ZJ);
    zp[2] = XSUB(XADD(XSUB(-ZI, H4), HA), ZJ);
    zp[3] = XSUB(XSUB(XADD(ZI, H2), HA), ZJ);
#pragma unroll
    for (int k = 0; k < 4; ++k) z2[k] = XMUL(zp[k], zp[k]);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (b >= NJJ) break;
      double a[4], f = 0., sa = 0.;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        // a select, not a branch: images closer than EPS contribute zero (the
        // reciprocal of a zero distance is computed and dropped)
        const double RRk = XADD(r2[b], z2[k]);
        const double ri0 = rsqrt(RRk);
        const double ri = RRk > T2 ? ri0 : 0.;
        f += ri;
        a[k] = ri * ri * ri;
        sa += a[k];
      }
      const double p0 = zp[0] * a[0], p1 = zp[1] * a[1], p2 = zp[2] * a[2], p3 = zp[3] * a[3];
      o.fs[b] += A * f;
      o.sa[b] += A * sa;
      o.m1[b] += A * ((p0 - p1) - (p2 - p3));
      o.m2[b] += A * ((p0 + p1) + (p2 + p3));
    }
  }
}

// --- Rankine part of one pair, both symmetry classes -------------------------
// Real parts of D+/- and S+/- (the wave pass adds the rest, and in finite
// depth the exponential images of the submerged-panel branch, fd_image_sums,
// evaluated once per unordered pair).
struct RealOut {
  double dp, dm, sp, sm;
};

template <bool FD>
NB_HD __forceinline__ void pair_rankine(const GreenCtx& g, const OmegaParams& om, const double* ambda,
                                             const double* ar, double XGI, double YGI, double ZGI, double XNI,
                                             double YNI, double ZNI, bool self, const PanelRec& P, RealOut& out) {
  RankineOut r;
  rankine<FD>(g, FD ? XMUL(2., om.h) : 0., XGI, YGI, ZGI, self, P, r);
  out.dp = r.VSXP * XNI + r.VSYP * YNI + r.VSZP * ZNI;
  out.dm = r.VSXM * XNI + r.VSYM * YNI + r.VSZM * ZNI;
  out.sp = r.FSP;
  out.sm = r.FSM;
}

// Wave sums of both reflections -> wave parts of D+/-, S+/- of one pair
// (collocation normal XNI, YNI, ZNI; source panel area `aire`).
template <bool FD>
NB_HD __forceinline__ void wave_combine(const OmegaParams& om, double aire, int NJJ, WaveJJ* w, double XNI,
                                             double YNI, double ZNI, PairOut& out) {
  if (NJJ == 1) w[1] = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
  // VNSINFD (:456-500) scales the wave sums by K A / 2pi^2, K A / 2pi (and K
  // again for gradients) with a minus sign; VNSFD (:830-865) adds them as they are
  double s1 = 1., s2 = 1., v1 = 1., v2 = 1.;
  if (!FD) {
    const double DPI = 2. * 3.141592653589793, DPI2 = 2. * 3.141592653589793 * 3.141592653589793;
    const double AKAIR = om.k0 * aire;
    const double ADPI2 = AKAIR / DPI2, ADPI = AKAIR / DPI;
    s1 = -ADPI2;
    s2 = -ADPI;
    v1 = -ADPI2 * om.k0;
    v2 = -ADPI * om.k0;
  }
  const double BM = (NJJ == 2) ? -1. : 1.;   // minus class: w0 - w1 (w1 = 0 without symmetry)
  const double SP1 = (w[0].FS1 + w[1].FS1) * s1, SM1 = (w[0].FS1 + BM * w[1].FS1) * s1;
  const double SP2 = (w[0].FS2 + w[1].FS2) * s2, SM2 = (w[0].FS2 + BM * w[1].FS2) * s2;
  const double VXP1 = (w[0].VSX1 + w[1].VSX1) * v1, VXM1 = (w[0].VSX1 + BM * w[1].VSX1) * v1;
  const double VYP1 = (w[0].VSY1 + w[1].VSY1) * v1, VYM1 = (w[0].VSY1 + BM * w[1].VSY1) * v1;
  const double VZP1 = (w[0].VSZ1 + w[1].VSZ1) * v1, VZM1 = (w[0].VSZ1 + BM * w[1].VSZ1) * v1;
  const double VXP2 = (w[0].VSX2 + w[1].VSX2) * v2, VXM2 = (w[0].VSX2 + BM * w[1].VSX2) * v2;
  const double VYP2 = (w[0].VSY2 + w[1].VSY2) * v2, VYM2 = (w[0].VSY2 + BM * w[1].VSY2) * v2;
  const double VZP2 = (w[0].VSZ2 + w[1].VSZ2) * v2, VZM2 = (w[0].VSZ2 + BM * w[1].VSZ2) * v2;
  out.dp_re = VXP1 * XNI + VYP1 * YNI + VZP1 * ZNI;
  out.dp_im = VXP2 * XNI + VYP2 * YNI + VZP2 * ZNI;
  out.dm_re = VXM1 * XNI + VYM1 * YNI + VZM1 * ZNI;
  out.dm_im = VXM2 * XNI + VYM2 * YNI + VZM2 * ZNI;
  out.sp_re = SP1;
  out.sp_im = SP2;
  out.sm_re = SM1;
  out.sm_im = SM2;
}

// --- wave part of one pair, both symmetry classes ----------------------------
template <bool FD>
NB_HD __forceinline__ void pair_wave(const GreenCtx& g, const OmegaParams& om, double XGI, double YGI, double ZGI,
                                          double XNI, double YNI, double ZNI, const PanelRec& P, PairOut& out) {
  const int NJJ = g.nsymy + 1;
  double ZMIII = ZGI;
  if (ZGI > g.zer) ZMIII = FD ? XMUL(20., g.zer) : g.zer;
  WaveJJ w[2];
  if ((ZGI < g.zer) && (P.zg < g.zer)) {
    if (FD) wave_fd_pair(g, om, XGI, YGI, ZMIII, P, NJJ, w);
    else wave_infd_pair(g, om, XGI, YGI, ZMIII, P, NJJ, w);
  } else {
#pragma unroll 1
    for (int JJ = 1; JJ <= NJJ; ++JJ) {
      if (FD) wave_fd_fs(om, XGI, YGI, ZMIII, JJ, P, w[JJ - 1]);
      else wave_infd_fs(om, XGI, YGI, ZMIII, JJ == 1 ? 1 : -1, P, w[JJ - 1]);
    }
  }
  wave_combine<FD>(om, P.aire, NJJ, w, XNI, YNI, ZNI, out);
}

}  // namespace nb200
