// CPU check of the assembly's pair functions (test infrastructure).
//
// The Rankine and wave functions that the assembly kernels call for each pair
// of panels (nemoh_b200/csrc/green.cuh and assembly.cuh) are compiled here for
// the host and applied the way the kernels apply them. Assembly: the Rankine and
// wave passes: the Rankine pass writes the real parts of D+/- and S+/- for every
// ordered pair (collocation I, source J); the wave pass takes each unordered
// pair I <= J once, evaluates both orders together when both panels are
// submerged and each order on its own otherwise, adds the results to the real
// parts and writes the imaginary parts. The per-frequency setup takes the same
// host functions as the library (fd_setup.cpp: X0, LISC, CINT, table nodes,
// stencil thresholds) in the order of SOLVE_BEM.f90:62-84; the tabulated wave
// integrals come from the caller (the oracle's CREK tables), since the
// library computes them with a kernel. Free surface: the field-point Green
// functions of every panel at every point, contracted with the source
// strengths as the free-surface kernel does, ETA = i W / G PHI. Kochin: the
// panel integrals of the Kochin kernel, contracted with the source strengths.
// The tests compare all three with the oracle's on the same mesh and
// frequencies. Pre-processor: the panel quantities and radiation conditions
// of the body-conditions kernel, compared with the pre-processor restatement.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../nemoh_b200/csrc/assembly.cuh"
#include "../../nemoh_b200/csrc/freesurface.cuh"
#include "../../nemoh_b200/csrc/kochin.cuh"
#include "../../nemoh_b200/csrc/preproc.cuh"
#include "../../nemoh_b200/csrc/fd_setup.h"

using namespace nb200;

namespace {

const double kPI = 4. * std::atan(1.);

// per-frequency parameters (SOLVE_BEM.f90:62-84, SOLVE_BEM_INFD_DIRECT.f90:79,
// SOLVE_BEM_FD_DIRECT.f90:99, COMPUTE_GREEN_FD.f90:259-268); 0 or a status code
int frequency_setup(double W, double g, double depth, double gm, int* nq_state, OmegaParams& om) {
  std::memset(&om, 0, sizeof om);
  om.w = W;
  om.h = depth;
  const double kwave = W * W / g;
  const bool fd = !((depth == 0.) || (kwave * depth >= 20));
  if (std::fabs(W) < 1.E-4) return ST_OMEGA;
  double qq[MAX_NQ + 2], cq[MAX_NQ + 2];
  if (!fd) {
    om.k0 = W * W / g;
    const int n = theta_quadrature(om.k0 * gm, qq, cq);
    om.nq = std::min(*nq_state, n);
    for (int i = 1; i <= om.nq; ++i) {
      om.cq[i] = cq[i];
      om.ct[i] = std::cos(qq[i]);
      om.st[i] = std::sin(qq[i]);
    }
    return 0;
  }
  om.fd = 1;
  double AMH;
  int st = finite_depth_root(W * W * depth / g, &AMH);
  if (st) return st;
  const double AKH = AMH * std::tanh(AMH), AM0 = AMH / depth;
  om.k0 = AM0;
  om.amh = AMH;
  *nq_state = theta_quadrature(AM0 * gm, qq, cq);
  int nexp = 0;
  st = exponential_fit(AKH, AMH, &nexp, om.ambda, om.ar);
  if (st) return st;
  om.nexp = nexp;
  om.ambda[nexp + 1] = 0.;
  om.ar[nexp + 1] = 2.;
  const double A = (AMH + AKH) * (AMH + AKH) / (depth * (AMH * AMH - AKH * AKH + AKH));
  const double ADPI2 = -A / (8. * kPI * kPI), ADPI = -A / (8 * kPI);
  om.coe1 = ADPI2 / AM0;
  om.coe2 = ADPI / AM0;
  om.coe3 = ADPI2;
  om.coe4 = ADPI;
  return 0;
}

// GM: largest horizontal node-pair distance including the y-mirror
// (SOLVE_BEM_INFD_DIRECT.f90:66-76)
double largest_distance(int np, int nsymy, const double* xyz) {
  double best = 0.;
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j) {
      const double dx = XSUB(xyz[3 * j], xyz[3 * i]);
      for (int jj = 0; jj <= nsymy; ++jj) {
        const double dy = XSUB(xyz[3 * i + 1], xyz[3 * j + 1] * (jj ? -1. : 1.));
        best = std::fmax(best, XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy))));
      }
    }
  return best;
}

// 3-node Lagrange stencils of one table axis: nodes and reciprocal denominators
void stencils(const double* x, int n, double* out) {
  for (int k = 2; k < n; ++k) {
    const double a = x[k - 1], b = x[k], c = x[k + 1];
    double* q = out + 8 * k;
    q[0] = a;
    q[1] = b;
    q[2] = c;
    q[3] = 1. / ((a - b) * (a - c));
    q[4] = 1. / ((b - c) * (b - a));
    q[5] = 1. / ((c - a) * (c - b));
  }
}

void put(double* m, long long q, double re, double im) {
  m[2 * q] = re;
  m[2 * q + 1] = im;
}

template <bool FD>
void assemble(const GreenCtx& g, const OmegaParams& om, const std::vector<PanelRec>& P, double* dp, double* dm,
              double* sp, double* sm) {
  const int N = (int)P.size(), NJJ = g.nsymy + 1;
  for (int J = 0; J < N; ++J)
    for (int I = 0; I < N; ++I) {
      RealOut r;
      pair_rankine<FD>(g, om, om.ambda, om.ar, P[I].xg, P[I].yg, P[I].zg, P[I].xn, P[I].yn, P[I].zn, I == J, P[J], r);
      const long long q = I + (long long)N * J;
      put(dp, q, r.dp, 0.);
      put(sp, q, r.sp, 0.);
      put(dm, q, r.dm, 0.);
      put(sm, q, r.sm, 0.);
    }
  auto add = [&](long long q, const PairOut& o) {
    put(dp, q, dp[2 * q] + o.dp_re, o.dp_im);
    put(sp, q, sp[2 * q] + o.sp_re, o.sp_im);
    put(dm, q, dm[2 * q] + o.dm_re, o.dm_im);
    put(sm, q, sm[2 * q] + o.sm_re, o.sm_im);
  };
  for (int J = 0; J < N; ++J)
    for (int I = 0; I <= J; ++I) {
      const PanelRec &PI = P[I], &PJ = P[J];
      const bool both = I != J;
      PairOut oij{}, oji{};
      if (PI.zg < g.zer && PJ.zg < g.zer) {
        if (FD) {
          if (!wave_fd_sym(g, om, PI, PJ, NJJ, both, oij, oji)) {
            set_status(g.status, ST_AKZ_UNDEFINED);
            oij = oji = PairOut{0, 0, 0, 0, 0, 0, 0, 0};
          }
          fd_images_pair(g, om, PI, PJ, NJJ, both, oij, oji);
        } else {
          wave_infd_both(g, om, PI, PJ, NJJ, both, oij, oji);
        }
      } else {
        pair_wave_ordered<FD>(g, om, PI, PJ, oij);
        if (both) pair_wave_ordered<FD>(g, om, PJ, PI, oji);
      }
      add(I + (long long)N * J, oij);
      if (both) add(J + (long long)N * I, oji);
    }
}

// Mesh, tables and Green-function context of one call
struct HostCtx {
  std::vector<PanelRec> P;
  std::vector<double> xr, xz, lag;
  std::vector<double4> tab;
  StencilThresholds thr;
  int status = 0;
  double gm = 0.;
  GreenCtx gc;

  HostCtx(int np, int nfa, int nsymy, const double* xyz, const int* m1234, const double* geo, double zer,
          const double* apd)
      : P(nfa), xr(TAB_IR + 2, 0.), xz(TAB_JZ + 2, 0.), lag(8 * (size_t)(TAB_IR + 2 + TAB_JZ + 2), 0.),
        tab((size_t)TAB_IR * TAB_JZ) {
    for (int i = 0; i < nfa; ++i) {
      PanelRec& p = P[i];
      p.xn = geo[0 * nfa + i];
      p.yn = geo[1 * nfa + i];
      p.zn = geo[2 * nfa + i];
      p.xg = geo[3 * nfa + i];
      p.yg = geo[4 * nfa + i];
      p.zg = geo[5 * nfa + i];
      p.aire = geo[6 * nfa + i];
      p.tdis = geo[7 * nfa + i];
      for (int v = 0; v < 4; ++v) {
        const int k = m1234[4 * i + v] - 1;
        p.vx[v] = xyz[3 * k];
        p.vy[v] = xyz[3 * k + 1];
        p.vz[v] = xyz[3 * k + 2];
      }
    }
    table_nodes(xr.data(), xz.data());
    for (size_t q = 0; q < tab.size(); ++q)
      tab[q] = make_double4(apd[q], apd[tab.size() + q], apd[2 * tab.size() + q], apd[3 * tab.size() + q]);
    stencils(xr.data(), TAB_IR, lag.data());
    stencils(xz.data(), TAB_JZ, lag.data() + 8 * (TAB_IR + 2));
    stencil_thresholds(&thr);
    double t = 1.E-8;   // largest double whose correctly rounded square root is <= 1e-4
    while (std::sqrt(std::nextafter(t, 1.)) <= 1.E-4) t = std::nextafter(t, 1.);
    while (std::sqrt(t) > 1.E-4) t = std::nextafter(t, 0.);
    gm = largest_distance(np, nsymy, xyz);
    gc.ro_eps2 = t;
    gc.xr = xr.data();
    gc.xz = xz.data();
    gc.apd = tab.data();
    gc.xlag = reinterpret_cast<const double4*>(lag.data());
    gc.zlag = reinterpret_cast<const double4*>(lag.data()) + 2 * (TAB_IR + 2);
    gc.thr = &thr;
    gc.zer = zer;
    gc.nsymy = nsymy;
    gc.status = &status;
  }
};

// ETA at the points for the source strengths of nprob problems (column-major
// nfa x nprob complex), as the free-surface kernel sums them
template <bool FD>
void free_surface(const GreenCtx& g, const OmegaParams& om, const std::vector<PanelRec>& P, double W, double grav,
                  int npts, const double* xy, int nprob, const double* zigb, const double* zigs, double* eta) {
  const int N = (int)P.size();
  for (int q = 0; q < npts; ++q)
    for (int p = 0; p < nprob; ++p) {
      double pot1 = 0., pot2 = 0.;
      for (int J = 0; J < N; ++J) {
        double SP1, SP2, SM1, SM2;
        field_green<FD>(g, om, xy[2 * q], xy[2 * q + 1], 0., P[J], SP1, SP2, SM1, SM2);
        const double bx = zigb[2 * ((size_t)p * N + J)], by = zigb[2 * ((size_t)p * N + J) + 1];
        if (g.nsymy == 0) {
          pot1 += bx * SP1 - by * SP2;
          pot2 += bx * SP2 + by * SP1;
        } else {
          const double sx = zigs[2 * ((size_t)p * N + J)], sy = zigs[2 * ((size_t)p * N + J) + 1];
          const double C1 = bx * (SP1 + SM1) + sx * (SP1 - SM1), D1 = by * (SP2 + SM2) + sy * (SP2 - SM2);
          const double C2 = bx * (SP2 + SM2) + sx * (SP2 - SM2), D2 = by * (SP1 + SM1) + sy * (SP1 - SM1);
          pot1 += (C1 - D1) * 0.5;
          pot2 += (C2 + D2) * 0.5;
        }
      }
      // ETA = i W / G PHI
      eta[2 * ((size_t)npts * p + q)] = -(W / grav) * pot2;
      eta[2 * ((size_t)npts * p + q) + 1] = (W / grav) * pot1;
    }
}

}  // namespace

// geo: 8 x nfa (XN, YN, ZN, XG, YG, ZG, AIRE, TDIS); m1234: 4 x nfa, 1-based;
// apd: {APD1X, APD1Z, APD2X, APD2Z} as 4 x 328 x 46 (column-major per table);
// nq_state: the reference's NQ, in and out. Outputs: complex n x n,
// column-major; without symmetry dm = dp and sm = sp. Returns 0 or a status.
extern "C" int host_pairs_assemble(int np, int nfa, int nsymy, const double* xyz, const int* m1234, const double* geo,
                                   double zer, const double* apd, double g, double depth, double omega,
                                   int* nq_state, int* fd_mode, double* dp, double* dm, double* sp, double* sm) {
  HostCtx h(np, nfa, nsymy, xyz, m1234, geo, zer, apd);
  OmegaParams om;
  const double T = 2. * kPI / omega;
  const int st = frequency_setup(2. * kPI / T, g, depth, h.gm, nq_state, om);
  if (st) return st;
  if (om.fd) assemble<true>(h.gc, om, h.P, dp, dm, sp, sm);
  else assemble<false>(h.gc, om, h.P, dp, dm, sp, sm);
  if (!nsymy) {   // one symmetry class: the library keeps D and S only
    std::memcpy(dm, dp, sizeof(double) * 2 * (size_t)nfa * nfa);
    std::memcpy(sm, sp, sizeof(double) * 2 * (size_t)nfa * nfa);
  }
  if (fd_mode) *fd_mode = om.fd;
  return h.status;
}

// Free-surface elevation at npts points (x, y, 0) (xy: npts x 2, row-major) of
// nprob problems solved at `period` (zigb, zigs: nfa x nprob complex; zigs
// unused without symmetry); eta: npts x nprob complex. The frequency setup
// leaves the NQ state as it is (nq_state is read only).
extern "C" int host_pairs_free_surface(int np, int nfa, int nsymy, const double* xyz, const int* m1234,
                                       const double* geo, double zer, const double* apd, double g, double depth,
                                       double period, int nq_state, int npts, const double* xy, int nprob,
                                       const double* zigb, const double* zigs, double* eta) {
  HostCtx h(np, nfa, nsymy, xyz, m1234, geo, zer, apd);
  OmegaParams om;
  const double W = 2. * kPI / period;
  int nq = nq_state;
  const int st = frequency_setup(W, g, depth, h.gm, &nq, om);
  if (st) return st;
  // COMPUTE_POTENTIAL_DOMAIN.f90:46: deep-water forms when Depth = 0 or AMH >= 20
  const double amh = om.fd ? om.amh : om.k0 * depth;
  const bool fd = !((depth == 0.) || (amh >= 20));
  if (fd) free_surface<true>(h.gc, om, h.P, W, g, npts, xy, nprob, zigb, zigs, eta);
  else free_surface<false>(h.gc, om, h.P, W, g, npts, xy, nprob, zigb, zigs, eta);
  return h.status;
}

// Kochin function H (ntheta x nprob complex) at the directions theta of
// nprob problems solved at `period` (COMPUTE_KOCHIN.f90:25-152 with the wave
// number of SOLVE_BEM.f90:62-84); yeff is taken as 0 on symmetric meshes.
extern "C" int host_pairs_kochin(int nfa, int nsymy, const double* xyz, const int* m1234, const double* geo,
                                 double g, double depth, double period, double xeff, double yeff, int ntheta,
                                 const double* theta, int nprob, const double* zigb, const double* zigs, double* h) {
  const double W = 2. * kPI / period;
  double kwave = W * W / g;
  if (!((depth == 0.) || (kwave * depth >= 20))) {
    double AMH;
    const int st = finite_depth_root(W * W * depth / g, &AMH);
    if (st) return st;
    kwave = AMH / depth;
  }
  const double ye = nsymy ? 0. : yeff;
  std::vector<double> rows(6 * (size_t)nfa);   // XG, YG, ZG, XN, YN, ZN
  for (int i = 0; i < nfa; ++i)
    for (int r = 0; r < 3; ++r) {
      rows[r * nfa + i] = geo[(3 + r) * nfa + i];
      rows[(3 + r) * nfa + i] = geo[r * nfa + i];
    }
  const double q = 0.25 / 3.141592653589793;
  for (int t = 0; t < ntheta; ++t) {
    const double ct = std::cos(theta[t]), st = std::sin(theta[t]);
    std::vector<cplx> zs(2 * (size_t)nfa);
    for (int i = 0; i < nfa; ++i) {
      zs[2 * i] = zs[2 * i + 1] = mk(0., 0.);
      kochin_panel(xyz, m1234, rows.data(), nfa, nsymy, kwave, depth, xeff, ye, ct, st, i, &zs[2 * i]);
    }
    for (int p = 0; p < nprob; ++p) {
      cplx acc = mk(0., 0.);
      for (int i = 0; i < nfa; ++i) {
        const size_t k = (size_t)p * nfa + i;
        acc = acc + mk(zigb[2 * k], zigb[2 * k + 1]) * zs[2 * i];
        if (nsymy) acc = acc + mk(zigs[2 * k], zigs[2 * k + 1]) * zs[2 * i + 1];
      }
      h[2 * ((size_t)ntheta * p + t)] = q * acc.re;
      h[2 * ((size_t)ntheta * p + t) + 1] = q * acc.im;
    }
  }
  return 0;
}

// Pre-processor panel quantities (centroid, normal, area: 7 x nfa) and the
// radiation condition n . d or n . (d x (x - axis)) of each DOF (ndof x nfa)
// for DOF specs (kind, dir[3], axis[3]) on a one-body mesh
extern "C" void host_pairs_preproc(int nfa, const double* xyz, const int* m1234, int ndof, const int* kind,
                                   const double* dir, const double* axis, double* panel, double* rad) {
  for (int i = 0; i < nfa; ++i) {
    double xm[3], n[3], area;
    pre_panel(xyz, m1234, i, xm, n, area);
    for (int c = 0; c < 3; ++c) {
      panel[c * nfa + i] = xm[c];
      panel[(3 + c) * nfa + i] = n[c];
    }
    panel[6 * nfa + i] = area;
    for (int d = 0; d < ndof; ++d) {
      PreDof q;
      q.kind = kind[d];
      q.body = 1;
      for (int c = 0; c < 3; ++c) {
        q.dir[c] = dir[3 * d + c];
        q.axis[c] = axis[3 * d + c];
      }
      rad[d * nfa + i] = pre_dof(q, xm, n);
    }
  }
}

// The wave pass's tile enumeration: for a T x T tile grid, the number of
// upper-triangle tiles (a <= b) that blocks 0 .. T(T+1)/2 - 1 do not map to
// exactly once (0 when every tile is taken by exactly one block)
extern "C" long long host_pairs_tri_tile_misses(int T) {
  std::vector<int> hits((size_t)T * T, 0);
  const long long nt = (long long)T * (T + 1) / 2;
  long long bad = 0;
  for (long long t = 0; t < nt; ++t) {
    int a, b;
    tri_tile((int)t, T, a, b);
    if (a < 0 || b < a || b >= T) ++bad;
    else ++hits[(size_t)a * T + b];
  }
  for (int a = 0; a < T; ++a)
    for (int b = a; b < T; ++b) bad += hits[(size_t)a * T + b] != 1;
  return bad;
}
