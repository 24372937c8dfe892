// Host-side per-frequency setup of the Nemoh BEM solve: scalar work that
// feeds the device kernels (no per-pair work happens here).
//
//  * dispersion root m0*h            X0    (Solver/Core/COMPUTE_GREEN_FD.f90:1635-1680)
//  * theta quadrature                CINT_INFD / CINT_FD (COMPUTE_GREEN_INFD.f90:505-638)
//  * finite-depth exponential fit    LISC with EXPORS, MCAS, SPRBM, SPQFB, HOUSRS, FF
//                                    (COMPUTE_GREEN_FD.f90:1007-1632)
//  * Green-table nodes XR, XZ        CREK (Solver/NEMOH.f90:179-199)
//  * exact stencil thresholds for the table lookups (COMPUTE_GREEN_INFD.f90:292-305)
//
// The arithmetic is evaluated in the same order as the reference (built with
// -ffp-contract=off), so these scalars are bit-identical to a double-precision
// run of the reference routines on the same machine.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fd_setup.h"

namespace nb200 {
namespace {

inline double sgnf(double a, double b) { return std::copysign(std::fabs(a), b); }
inline double sq(double x) { return x * x; }

// column-major work matrix with the reference's leading dimension 4*(31-1)
struct WorkMat {
  static constexpr int LDA = 120;
  double v[LDA * 32];
  double& operator()(int i, int j) { return v[(i - 1) + LDA * (j - 1)]; }
};

struct SetupError {
  int code;
};

// Householder least squares, solution in the right-hand-side columns
void housrs(WorkMat& A, int rows, int cols, int nrhs, double eps) {
  const int ntc = cols + nrhs;
  if (cols > rows) throw SetupError{ST_HOUSRS};
  for (int k = 1; k <= cols; ++k) {
    double e = 0;
    for (int i = k; i <= rows; ++i) e = e + sq(A(i, k));
    const double e0 = std::sqrt(e);
    if (e0 < eps) throw SetupError{ST_HOUSRS};
    const double akk = A(k, k);
    const double alpha = (akk == 0) ? -e0 : -sgnf(e0, akk);
    const double eta = alpha * (alpha - akk);
    for (int j = k + 1; j <= ntc; ++j) {
      double ba = (A(k, k) - alpha) * A(k, j);
      for (int i = k + 1; i <= rows; ++i) ba = ba + A(i, k) * A(i, j);
      A(k, j) = A(k, j) + ba / alpha;
      for (int i = k + 1; i <= rows; ++i) A(i, j) = A(i, j) - A(i, k) * ba / eta;
    }
    A(k, k) = alpha;
    for (int i = k + 1; i <= rows; ++i) A(i, k) = 0;
  }
  for (int j = 1; j <= nrhs; ++j) {
    const int c = cols + j;
    A(cols, c) = A(cols, c) / A(cols, cols);
    for (int l = 2; l <= cols; ++l) {
      const int i1 = cols + 1 - l;
      for (int i = i1 + 1; i <= cols; ++i) A(i1, c) = A(i1, c) - A(i1, i) * A(i, c);
      A(i1, c) = A(i1, c) / A(i1, i1);
    }
  }
}

// Bairstow quadratic-factor iteration (SPQFB). Returns its status flag.
int quadratic_factor(double* C, int ic, double* Q, int lim) {
  int I, J, L, LL, ier = 0;
  double H = 0., HH = 0., A, A1, AA, B, BB, B1, C1 = 0., CA, CB, CC, CD, DQ1, DQ2;
  double Q1, Q2, QQ1, QQ2, QQQ1, QQQ2;
  const double EPS = 1.E-14, EPS1 = 1.E-6;
  J = ic + 1;
s1:
  J = J - 1;
  if (J - 1 <= 0) return -1;
  if (C[J] == 0) goto s1;
  A = C[J];
  if (A - 1. != 0) {
    for (I = 1; I <= J; ++I) {
      C[I] = C[I] / A;
      if (std::fabs(C[I]) - 1.E27 >= 0) return -1;
    }
  }
  if (J - 3 < 0) return -2;
  if (J - 3 == 0) {
    Q[1] = C[1]; Q[2] = C[2]; Q[3] = 0.; Q[4] = 0.;
    return 0;
  }
restart:
  L = 0;
  LL = 0;
  Q1 = Q[1];
  Q2 = Q[2];
  QQ1 = 0.;
  QQ2 = 0.;
  AA = C[1];
  BB = C[2];
  CB = std::fabs(AA);
  CA = std::fabs(BB);
  if (CB - CA < 0) { CC = CB + CB; CB = CB / CA; CA = 1.; }
  else if (CB - CA == 0) { CC = CA + CA; CA = 1.; CB = 1.; }
  else { CC = CA + CA; CA = CA / CB; CB = 1.; }
  CD = CC * .1;
iterate:
  A = 0.;
  B = A;
  A1 = A;
  B1 = A;
  I = J;
  QQQ1 = Q1;
  QQQ2 = Q2;
  DQ1 = HH;
  DQ2 = H;
  for (;;) {
    H = -Q1 * B - Q2 * A + C[I];
    if (std::fabs(H) - 1.E27 >= 0) goto diverged;
    B = A;
    A = H;
    I = I - 1;
    if (I - 1 < 0) break;
    if (I - 1 == 0) H = 0.;
    H = -Q1 * B1 - Q2 * A1 + H;
    if (std::fabs(H) - 1.E27 >= 0) goto diverged;
    C1 = B1;
    B1 = A1;
    A1 = H;
  }
  H = CA * std::fabs(A) + CB * std::fabs(B);
  if (LL > 0) goto converged;
  L = L + 1;
  if (!(std::fabs(A) - EPS * std::fabs(C[1]) > 0) && !(std::fabs(B) - EPS * std::fabs(C[2]) > 0)) goto converged;
  if (H - CC <= 0) {
    AA = A; BB = B; CC = H; QQ1 = Q1; QQ2 = Q2;
  }
  if (L - lim > 0) {
    if (H - CD <= 0) { ier = 1; goto best; }
    if (Q[1] == 0 && Q[2] == 0) goto diverged;
    Q[1] = 0.;
    Q[2] = 0.;
    goto restart;
  }
  HH = std::fmax(std::fmax(std::fabs(A1), std::fabs(B1)), std::fabs(C1));
  if (HH <= 0) goto diverged;
  A1 = A1 / HH;
  B1 = B1 / HH;
  C1 = C1 / HH;
  H = A1 * C1 - B1 * B1;
  if (H == 0) goto diverged;
  A = A / HH;
  B = B / HH;
  HH = (B * A1 - A * B1) / H;
  H = (A * C1 - B * B1) / H;
  Q1 = Q1 + HH;
  Q2 = Q2 + H;
  if (!(std::fabs(HH) - EPS * std::fabs(Q1) > 0) && !(std::fabs(H) - EPS * std::fabs(Q2) > 0)) {
    LL = 1;
    goto iterate;
  }
  if (L - 1 <= 0) goto iterate;
  if (std::fabs(HH) - EPS1 * std::fabs(Q1) > 0) goto iterate;
  if (std::fabs(H) - EPS1 * std::fabs(Q2) > 0) goto iterate;
  if (std::fabs(QQQ1 * HH) - std::fabs(Q1 * DQ1) >= 0) goto best;
  if (std::fabs(QQQ2 * H) - std::fabs(Q2 * DQ2) < 0) goto iterate;
  goto best;
converged:
  Q[1] = Q1; Q[2] = Q2; Q[3] = A; Q[4] = B;
  return ier;
diverged:
  ier = -3;
best:
  Q[1] = QQ1; Q[2] = QQ2; Q[3] = AA; Q[4] = BB;
  return ier;
}

// All roots of the real polynomial C(1..ic) (SPRBM). Roots in rr/rc.
void polynomial_roots(double* C, int ic, double* rr, double* rc, double* pol) {
  int I, J, L, N, IR, IST = 1, ier = 0;
  double A, B, H, Q1, Q2, Q[5];
  const int LIM = 100;
  IR = ic + 1;
  do {
    IR = IR - 1;
    if (IR - 1 <= 0) throw SetupError{ST_SPRBM};
  } while (C[IR] == 0);
  J = IR;
  L = 0;
  A = C[IR];
  for (I = 1; I <= IR; ++I) {
    if (L <= 0) {
      if (C[I] == 0) {
        rr[I] = 0.; rc[I] = 0.; pol[J] = 0.;
        J = J - 1;
        continue;
      }
      L = 1;
      IST = I;
      J = 0;
    }
    J = J + 1;
    C[I] = C[I] / A;
    pol[J] = C[I];
    if (std::fabs(pol[J]) - 1.E27 >= 0) throw SetupError{ST_SPRBM};
  }
  Q1 = 0.;
  Q2 = 0.;
  for (;;) {
    if (J - 2 < 0) {
      IR = IR - 1;
      break;
    }
    if (J - 2 == 0) {
      A = pol[1];
      rr[IST] = -A;
      rc[IST] = 0.;
      IR = IR - 1;
      Q2 = 0.;
      if (IR - 1 > 0) {
        for (I = 2; I <= IR; ++I) {
          Q1 = Q2;
          Q2 = pol[I + 1];
          pol[I] = A * Q2 + Q1;
        }
      }
      pol[IR + 1] = A + Q2;
      break;
    }
    bool found = false;
    for (L = 1; L <= 10 && !found; ++L) {
      N = 1;
      for (;;) {
        Q[1] = Q1;
        Q[2] = Q2;
        int st = quadratic_factor(pol, J, Q, LIM);
        if (st >= 0) {
          if (st > 0) ier = 1;
          found = true;
          break;
        }
        if (Q1 == 0 && Q2 == 0) N = 4;
        if (N == 1 || N == 3) { Q1 = -Q1; N = N + 1; continue; }
        if (N == 2) { Q2 = -Q2; N = N + 1; continue; }
        Q1 = 1. + Q1;
        Q2 = 1. - Q2;
        break;
      }
    }
    if (!found) {
      // IER=3: no quadratic factor after 10 restarts; the reference returns
      // with the roots found so far (and no error stop)
      return;
    }
    Q1 = Q[1];
    Q2 = Q[2];
    B = 0.;
    A = 0.;
    I = J;
    do {
      H = -Q1 * B - Q2 * A + pol[I];
      pol[I] = B;
      B = A;
      A = H;
      I = I - 1;
    } while (I - 2 > 0);
    pol[2] = B;
    pol[1] = A;
    L = IR - 1;
    if (J - L <= 0)
      for (I = J; I <= L; ++I) pol[I - 1] = pol[I - 1] + pol[I] * Q2 + pol[I + 1] * Q1;
    pol[L] = pol[L] + pol[L + 1] * Q2 + Q1;
    pol[IR] = pol[IR] + Q2;
    H = -.5 * Q2;
    A = H * H - Q1;
    B = std::sqrt(std::fabs(A));
    if (A <= 0) {
      rr[IST] = H; rc[IST] = B;
      IST = IST + 1;
      rr[IST] = H; rc[IST] = -B;
    } else {
      B = H + sgnf(B, H);
      rr[IST] = Q1 / B; rc[IST] = 0.;
      IST = IST + 1;
      rr[IST] = B; rc[IST] = 0.;
    }
    IST = IST + 1;
    J = J - 2;
  }
  A = 0.;
  for (I = 1; I <= IR; ++I) {
    Q1 = C[I];
    Q2 = pol[I + 1];
    pol[I] = Q2;
    if (Q1 != 0) Q2 = (Q1 - Q2) / Q1;
    Q2 = std::fabs(Q2);
    if (Q2 - A > 0) A = Q2;
  }
  I = IR + 1;
  pol[I] = 1.;
  rr[I] = A;
  rc[I] = 0.;
  (void)ier;
}

// function fitted by the exponential sum (FF)
double fit_target(double x, double ak, double am) {
  const double coef = sq(am + ak) / (sq(am) - sq(ak) + ak);
  const double tol = std::fmax(0.1, 0.1 * am);
  if (std::fabs(x - am) > tol)
    return (x + ak) * std::exp(x) / (x * std::sinh(x) - ak * std::cosh(x)) - coef / (x - am) - 2.;
  const double a = am - tol, b = am, c = am + tol;
  const double d = (a + ak) * std::exp(a) / (a * std::sinh(a) - ak * std::cosh(a)) - coef / (a - am) - 2;
  const double e = coef / (am + ak) * (am + ak + 1) - sq(coef / (am + ak)) * am - 2;
  const double f = (c + ak) * std::exp(c) / (c * std::sinh(c) - ak * std::cosh(c)) - coef / (c - am) - 2;
  return (x - b) * (x - c) * d / ((a - b) * (a - c)) + (x - c) * (x - a) * e / ((b - c) * (b - a)) +
         (x - a) * (x - b) * f / ((c - a) * (c - b));
}

// Prony fit (EXPORS + MCAS): exponents into lam[1..nm], amplitudes amp[1..nm]
void prony_fit(const double* xt, const double* yt, int nj, int& nm, double* lam, double* amp, WorkMat& S) {
  const int npp = nj + 1;
  const double h = (xt[npp] - xt[1]) / nj;
  const int rows = npp - nm;
  for (int i = 1; i <= rows; ++i) {
    for (int j = 1; j <= nm; ++j) S(i, j) = yt[nm - j + i];
    S(i, nm + 1) = -yt[nm + i];
  }
  housrs(S, rows, nm, 1, 1.E-20);
  double sc[33] = {0}, vr[33] = {0}, vc[33] = {0}, pol[33] = {0};
  for (int i = 1; i <= nm; ++i) sc[nm - i + 1] = S(i, nm + 1);
  sc[nm + 1] = 1.;
  polynomial_roots(sc, nm + 1, vr, vc, pol);
  for (int i = 1; i <= nm; ++i) {
    std::complex<double> z = std::log(std::complex<double>(vr[i], vc[i])) / h;
    vr[i] = z.real();
    vc[i] = z.imag();
  }
  int i = 1, j = 0;
  do {
    j = j + 1;
    lam[j] = vr[i];
    if (vc[i] != 0 && std::fabs(vr[i] - vr[i + 1]) - 1.E-5 <= 0) i = i + 2;
    else i = i + 1;
  } while (i - nm <= 0);
  int nexp = j;
  j = 0;
  for (i = 1; i <= nexp; ++i) {
    if (lam[i] >= 0. || lam[i] + 20. <= 0) continue;
    ++j;
    lam[j] = lam[i];
  }
  nexp = j;
  nm = nexp;
  // least-squares amplitudes for the retained exponents (MCAS)
  for (int a = 1; a <= nexp; ++a)
    for (int b = 1; b <= nexp; ++b) {
      double s = 0;
      for (int l = 1; l <= npp; ++l) {
        const double t = (lam[a] + lam[b]) * xt[l];
        if (t + 30 >= 0) s = s + std::exp(t);
      }
      S(a, b) = s;
    }
  for (int a = 1; a <= nexp; ++a) {
    double s = 0;
    for (int l = 1; l <= npp; ++l) {
      const double t = lam[a] * xt[l];
      if (t + 30 >= 0) s = s + std::exp(t) * yt[l];
    }
    S(a, nexp + 1) = s;
  }
  housrs(S, nexp, nexp, 1, 1.E-20);
  for (int a = 1; a <= nexp; ++a) amp[a] = S(a, nexp + 1);
}

}  // namespace

double preproc_wavenumber(double w, double g, double depth) {
  double k = w * w / g;
  const double x0 = k * depth;
  if (x0 > 0. && x0 <= 20.) {
    double xg = 0., xd = x0;
    int nite = 0;
    while (nite < 10000 && (x0 - xg * std::tanh(xg)) * (x0 - xd * std::tanh(xd)) > 0.) {
      xg = xd;
      xd = 2. * xd;
      ++nite;
    }
    nite = 0;
    double xc = 0.5 * (xd + xg);
    while (nite < 10000 && std::fabs(xd - xg) / std::fabs(xc) >= 1.0e-6) {
      xc = 0.5 * (xd + xg);
      if ((x0 - xg * std::tanh(xg)) * (x0 - xc * std::tanh(xc)) > 0.) xg = xc;
      else xd = xc;
      ++nite;
    }
    k = xc / depth;
  }
  return k;
}

int finite_depth_root(double ak, double* out) {
  const double EPS = 5.E-6;
  int itour = 0, iiter = 0;
  double xi = 0., xs = xi, xm;
  const double pas = std::fmax(ak, std::sqrt(ak));
  do {
    xs = xs + pas;
    itour = itour + 1;
    if (itour > 1000) break;
  } while ((ak - xs * std::tanh(xs)) * (ak - xi * std::tanh(xi)) > 0);
  for (;;) {
    xm = (xi + xs) * 0.5;
    iiter = iiter + 1;
    if (iiter > 1000 || itour > 1000) return ST_DISPERSION;
    if (!(std::fabs((xs - xi) / xm) > EPS)) break;
    double v1 = ak - xm * std::tanh(xm);
    const double v2 = ak - xi * std::tanh(xi);
    if (std::fabs(v1 * v2) <= 1.E-12) v1 = 0.;
    if (v1 * v2 < 0) xs = xm;
    else xi = xm;
  }
  *out = xm;
  return ST_OK;
}

int exponential_fit(double akh, double amh, int* nexp, double* ambda, double* ar) {
  try {
    static thread_local WorkMat S;
    std::memset(S.v, 0, sizeof S.v);
    for (int i = 0; i <= MAX_NEXP; ++i) ar[i] = 0.;
    double xt[122] = {0}, yt[122] = {0};
    const double A = -0.1, B = 20., PRECI = 1.E-02, NEXR = 31;
    int nk = 4, nm = 0;
    for (;;) {
      nm = nk;
      const int nj = 4 * nm, npp = nj + 1;
      const double h = (B - A) / nj;
      for (int i = 1; i <= npp; ++i) {
        xt[i] = A + (i - 1) * h;
        yt[i] = fit_target(xt[i], akh, amh);
      }
      prony_fit(xt, yt, nj, nm, ambda, ar, S);
      const int nmo = 2 * npp - 2 + 1;
      bool miss = false;
      for (int i = 1; i <= nmo; ++i) {
        const double xx = (i - 1) * B / (nmo - 1);
        const double yy = fit_target(xx, akh, amh);
        double tt = 0.;
        for (int j = 1; j <= nm; ++j) {
          const double rt = ambda[j] * xx;
          if (rt > -20.) tt = tt + ar[j] * std::exp(rt);
        }
        if (std::fabs(yy - tt) > PRECI) miss = true;
      }
      if (!miss) break;
      nk = nk + 2;
      if (nk - (NEXR - 1) > 0) break;
    }
    for (int j = 1; j <= nm; ++j)
      if (ambda[j] > 0.) return ST_LISC;
    *nexp = nm;
    return ST_OK;
  } catch (const SetupError& e) {
    return e.code;
  }
}

static const double kQ8[4] = {.4801449, .3983332, .2627662, .09171732};
static const double kC8[4] = {.05061427, .1111905, .1568533, .1813419};
static const double kQ12[6] = {.4907803, .4520586, .3849513, .2936589, .1839157, .06261670};
static const double kC12[6] = {.2358766E-1, .5346966E-1, .8003916E-1, .1015837, .1167462, .1245735};
static const double kQ16[8] = {.4947004, .4722875, .4328156, .3777022, .3089381, .2290084, .1408017, .04750625};
static const double kC16[8] = {.01357622, .03112676, .04757925, .06231448, .07479799, .08457826, .09130170, .09472530};
static const double kQ24[12] = {.4975936, .4873642, .469137, .4432077, .4100009, .3700621,
                                .3240468, .2727107, .2168967, .1575213, .09555943, .032028446};
static const double kC24[12] = {.6170615E-2, .1426569E-1, .2213872E-1, .2964929E-1, .366732E-1, .4309508E-1,
                                .4880932E-1, .5372213E-1, .5775283E-1, .6083523E-1, .6291873E-1, .6396909E-1};
static const double kQ32[16] = {.4986319, .4928057, .4823811, .4674530, .4481605, .4246838, .3972418, .3660910,
                                .3315221, .2938578, .2534499, .2106756, .1659343, .1196436, .07223598, .02415383};
static const double kC32[16] = {.350930E-2, .8137197E-2, .1269603E-1, .1713693E-1, .2141794E-1, .2549903E-1,
                                .2934204E-1, .3291111E-1, .3617289E-1, .3909694E-1, .4165596E-1, .4382604E-1,
                                .4558693E-1, .4692219E-1, .4781936E-1, .4827004E-1};

int theta_quadrature(double akk, double* qq, double* cq) {
  const double PI = 4. * std::atan(1.);
  const double *q = nullptr, *c = nullptr;
  int n = 0, half = 0;
  if (akk <= .4) { n = 8; q = kQ8; c = kC8; half = 4; }
  else if (akk <= 2.5) { n = 12; q = kQ12; c = kC12; half = 6; }
  else if (akk <= 4.) { n = 16; q = kQ16; c = kC16; half = 8; }
  else if (akk <= 8.) { n = 24; q = kQ24; c = kC24; half = 12; }
  else if (akk <= 25.) { n = 32; q = kQ32; c = kC32; half = 16; }
  if (q) {
    for (int i = 1; i <= half; ++i) {
      qq[i] = q[i - 1] * PI;
      qq[n + 1 - i] = -q[i - 1] * PI;
      cq[i] = c[i - 1] * PI;
      cq[n + 1 - i] = c[i - 1] * PI;
    }
    return n;
  }
  n = (akk > 40.) ? 101 : 51;
  for (int j = 1; j <= n; ++j) {
    qq[j] = -PI / 2. + (j - 1.) / (n - 1.) * PI;
    if (j == 1 || j == n) cq[j] = PI / (3. * (n - 1.));
    else if (j % 2 != 0) cq[j] = 2. / (3. * (n - 1.)) * PI;
    else cq[j] = 4. / (3. * (n - 1.)) * PI;
  }
  return n;
}

void table_nodes(double* xr, double* xz) {
  for (int j = 1; j <= TAB_JZ; ++j)
    xz[j] = -std::fmin(std::fmin(std::pow(10., j / 5. - 6), std::pow(10., j / 8. - 4.5)), 16.);
  xr[1] = 0.;
  for (int i = 2; i <= TAB_IR; ++i) {
    if (i < 40) xr[i] = std::fmin(std::pow(10., (i - 1.) / 5 - 6), 4. / 3. + std::fabs((i - 32.) / 3.));
    else xr[i] = 4. / 3. + std::fabs((i - 32.) / 3.);
  }
}

void simpson_251(double* cqt, double* qqt) {
  const double PI = 4. * std::atan(1.);
  const int n = NPINTE;
  for (int j = 1; j <= n; ++j) {
    qqt[j] = -PI / 2. + (j - 1.) / (n - 1.) * PI;
    if (j == 1 || j == n) cqt[j] = PI / (3. * (n - 1.));
    else if (j % 2 != 0) cqt[j] = 2. / (3. * (n - 1.)) * PI;
    else cqt[j] = 4. / (3. * (n - 1.)) * PI;
  }
}

// smallest positive double x with f(x) >= k, for a monotone f (bisection on the bit pattern)
template <class F>
static double threshold(F f, int k, double lo, double hi) {
  if (f(lo) >= k) return -INFINITY;
  if (f(hi) < k) return INFINITY;
  uint64_t a, b;
  std::memcpy(&a, &lo, 8);
  std::memcpy(&b, &hi, 8);
  while (b - a > 1) {
    uint64_t m = a + (b - a) / 2;
    double x;
    std::memcpy(&x, &m, 8);
    if (f(x) >= k) b = m;
    else a = m;
  }
  double x;
  std::memcpy(&x, &b, 8);
  return x;
}

void stencil_thresholds(StencilThresholds* t) {
  auto f8 = [](double x) { return (int)(8 * (std::log10(x) + 4.5)); };
  auto f5 = [](double x) { return (int)(5 * (std::log10(x) + 6)); };
  auto fi = [](double y) { return (int)(5 * (std::log10(y) + 6) + 1); };
  for (int k = 0; k < 48; ++k) {
    t->kj8[k] = threshold(f8, k, 1.E-2, 16.);
    t->kj5[k] = threshold(f5, k, 1.E-7, 1.E-2);
    t->ki5[k] = threshold(fi, k, 1.E-20, 1.);
  }
}

}  // namespace nb200
