// Geometry, Green-table and influence-matrix assembly kernels (sm_100a, FP64).
#pragma once
#include "green.cuh"

namespace nb200 {

// ---------------------------------------------------------------------------
// GOMG (Solver/Core/PREPARE_MESH.f90:80-180): one thread per panel.
// Every operation is exactly rounded so that the panel geometry matches an
// FP64 CPU run of the reference bit for bit (it feeds every branch later).
// Writes the source-panel records and the collocation SoA rows
// (XG, YG, ZG, XN, YN, ZN) and flags degenerate panels.
// ---------------------------------------------------------------------------
__global__ void gomg_kernel(int nfa, const double* __restrict__ xyz, const int* __restrict__ m1234,
                            PanelRec* __restrict__ rec, double* __restrict__ rows, int* status) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nfa) return;
  const int K = m1234[4 * I] - 1, L = m1234[4 * I + 1] - 1, M = m1234[4 * I + 2] - 1, N = m1234[4 * I + 3] - 1;
  const double xk = xyz[3 * K], yk = xyz[3 * K + 1], zk = xyz[3 * K + 2];
  const double xl = xyz[3 * L], yl = xyz[3 * L + 1], zl = xyz[3 * L + 2];
  const double xm = xyz[3 * M], ym = xyz[3 * M + 1], zm = xyz[3 * M + 2];
  const double xn = xyz[3 * N], yn = xyz[3 * N + 1], zn = xyz[3 * N + 2];
  const double T1X = XSUB(xm, xk), T1Y = XSUB(ym, yk), T1Z = XSUB(zm, zk);
  const double T2X = XSUB(xn, xl), T2Y = XSUB(yn, yl), T2Z = XSUB(zn, zl);
  const double XNX = XSUB(XMUL(T1Y, T2Z), XMUL(T2Y, T1Z));
  const double XNY = XSUB(XMUL(T1Z, T2X), XMUL(T2Z, T1X));
  const double XNZ = XSUB(XMUL(T1X, T2Y), XMUL(T2X, T1Y));
  const double XNQ = XSQRT(XADD(XADD(XMUL(XNX, XNX), XMUL(XNY, XNY)), XMUL(XNZ, XNZ)));
  if (XNQ <= 1.E-25) {
    set_status(status, ST_PANEL_AREA);
    return;
  }
  const double NX = XDIV(XNX, XNQ), NY = XDIV(XNY, XNQ), NZ = XDIV(XNZ, XNQ);
  const double XAV = XMUL(XADD(XADD(XADD(xk, xm), xl), xn), 0.25);
  const double YAV = XMUL(XADD(XADD(XADD(yk, ym), yn), yl), 0.25);
  const double ZAV = XMUL(XADD(XADD(XADD(zk, zm), zn), zl), 0.25);
  const double T1 = XSQRT(XADD(XADD(XMUL(T1X, T1X), XMUL(T1Y, T1Y)), XMUL(T1Z, T1Z)));
  const double U1X = XDIV(T1X, T1), U1Y = XDIV(T1Y, T1), U1Z = XDIV(T1Z, T1);
  const double U2X = XSUB(XMUL(NY, U1Z), XMUL(NZ, U1Y));
  const double U2Y = XSUB(XMUL(NZ, U1X), XMUL(NX, U1Z));
  const double U2Z = XSUB(XMUL(NX, U1Y), XMUL(NY, U1X));
  auto proj = [&](double ux, double uy, double uz, double px, double py, double pz) {
    return XADD(XADD(XMUL(ux, XSUB(px, XAV)), XMUL(uy, XSUB(py, YAV))), XMUL(uz, XSUB(pz, ZAV)));
  };
  const double XI1 = proj(U1X, U1Y, U1Z, xk, yk, zk), XI2 = proj(U1X, U1Y, U1Z, xl, yl, zl);
  const double XI3 = proj(U1X, U1Y, U1Z, xm, ym, zm), XI4 = proj(U1X, U1Y, U1Z, xn, yn, zn);
  const double ETA1 = proj(U2X, U2Y, U2Z, xk, yk, zk), ETA2 = proj(U2X, U2Y, U2Z, xl, yl, zl);
  const double ETA3 = proj(U2X, U2Y, U2Z, xm, ym, zm), ETA4 = proj(U2X, U2Y, U2Z, xn, yn, zn);
  const double XIO = XDIV(XADD(XMUL(XI4, XSUB(ETA1, ETA2)), XMUL(XI2, XSUB(ETA4, ETA1))),
                          XMUL(3., XSUB(ETA2, ETA4)));
  const double ETAO = XDIV(-ETA1, 3.);
  const double EN1 = XSUB(ETA1, ETAO), EN2 = XSUB(ETA2, ETAO), EN3 = XSUB(ETA3, ETAO), EN4 = XSUB(ETA4, ETAO);
  const double XN1 = XSUB(XI1, XIO), XN2 = XSUB(XI2, XIO), XN3 = XSUB(XI3, XIO), XN4 = XSUB(XI4, XIO);
  PanelRec p;
  p.xg = XADD(XADD(XAV, XMUL(U1X, XIO)), XMUL(U2X, ETAO));
  p.yg = XADD(XADD(YAV, XMUL(U1Y, XIO)), XMUL(U2Y, ETAO));
  p.zg = XADD(XADD(ZAV, XMUL(U1Z, XIO)), XMUL(U2Z, ETAO));
  p.xn = NX;
  p.yn = NY;
  p.zn = NZ;
  p.aire = XMUL(XMUL(XSUB(XN3, XN1), XSUB(EN4, EN2)), 0.5);
  const double TT1 = XSQRT(XADD(XMUL(XN1, XN1), XMUL(EN1, EN1)));
  const double TT2 = XSQRT(XADD(XMUL(XN2, XN2), XMUL(EN2, EN2)));
  const double TT3 = XSQRT(XADD(XMUL(XN3, XN3), XMUL(EN3, EN3)));
  const double TT4 = XSQRT(XADD(XMUL(XN4, XN4), XMUL(EN4, EN4)));
  p.tdis = fmax(fmax(TT1, TT2), fmax(TT3, TT4));
  p.vx[0] = xk; p.vy[0] = yk; p.vz[0] = zk;
  p.vx[1] = xl; p.vy[1] = yl; p.vz[1] = zl;
  p.vx[2] = xm; p.vy[2] = ym; p.vz[2] = zm;
  p.vx[3] = xn; p.vy[3] = yn; p.vz[3] = zn;
  rec[I] = p;
  rows[0 * nfa + I] = p.xg;
  rows[1 * nfa + I] = p.yg;
  rows[2 * nfa + I] = p.zg;
  rows[3 * nfa + I] = p.xn;
  rows[4 * nfa + I] = p.yn;
  rows[5 * nfa + I] = p.zn;
}

// GM: largest horizontal node-pair distance including the y-mirror
// (SOLVE_BEM_INFD_DIRECT.f90:66-76). Non-negative doubles order like their
// bit patterns, so an unsigned atomicMax reduces them exactly.
__global__ void gm_kernel(int np, int nsymy, const double* __restrict__ xyz, unsigned long long* gm_bits) {
  double best = 0.;
  const long long total = (long long)np * np;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / np), j = (int)(q % np);
    if (j <= i) continue;
    const double dx = XSUB(xyz[3 * j], xyz[3 * i]);
    for (int jj = 0; jj <= nsymy; ++jj) {
      const double bj = jj ? -1. : 1.;
      const double dy = XSUB(xyz[3 * i + 1], xyz[3 * j + 1] * bj);
      best = fmax(best, XSQRT(XADD(XMUL(dx, dx), XMUL(dy, dy))));
    }
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(gm_bits, (unsigned long long)__double_as_longlong(best));
}

// ---------------------------------------------------------------------------
// CREK / VNS (Solver/NEMOH.f90:179-251): one thread per table node,
// 251-point Simpson rule in theta. cos(theta) comes from the host.
// ---------------------------------------------------------------------------
__global__ void crek_kernel(const double* __restrict__ xr, const double* __restrict__ xz,
                            const double* __restrict__ cqt, const double* __restrict__ ctt, double4* __restrict__ apd) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= TAB_IR * TAB_JZ) return;
  const int I = q % TAB_IR + 1, J = q / TAB_IR + 1;
  const double AKZ = xz[J], AKR = xr[I];
  double f1x = 0., f1z = 0., f2x = 0., f2z = 0.;
  for (int it = 1; it <= NPINTE; ++it) {
    const double CT = ctt[it], CQ = cqt[it];
    const cplx Z = mk(AKZ, XMUL(AKR, CT));
    const cplx CEX = (AKZ + 30. <= 0.) ? mk(0., 0.) : cexp_(Z);
    const cplx G = GG(Z, CEX);
    const cplx C1 = CQ * (G - 1. / Z);
    const cplx C2 = CQ * CEX;
    f1x += CT * C1.im;
    f1z += C1.re;
    f2x += CT * C2.im;
    f2z += C2.re;
  }
  apd[(I - 1) + TAB_IR * (J - 1)] = make_double4(f1x, f1z, f2x, f2z);
}

// ---------------------------------------------------------------------------
// Influence-matrix assembly. Thread = collocation row I, block = 128 rows;
// the block stages ASM_TJ source panels J in shared memory and walks them.
// Output per frequency (column-major, leading dimension N): D+ then D- in
// out.d, S+ then S- in out.s (nsymy=0: one D and one S). Column-major writes
// by consecutive rows are coalesced 16-byte stores.
//   rankine_cache_kernel: Rankine part (VAVINFD / VAVFD) of every pair. It
//                   depends on the geometry and the depth regime only (the
//                   seabed image at 2h in finite depth), not on the
//                   frequency, so it is evaluated once per mesh and regime
//                   into a real cache: (D+, S+) pairs, then (D-, S-).
//   rankine_kernel: the same Rankine part per frequency slot, written to the
//                   real parts (imaginary = 0) of the slot's matrices; used
//                   for resident bodies whose cache does not fit.
//   wave_sym_kernel: wave part (VNSINFD / VNSFD; in finite depth with the
//                   exponential images) added to the Rankine part (from the
//                   cache, or from the real parts the per-slot pass wrote) and
//                   written to both parts of the matrices; in mixed precision
//                   it also writes the FP32 copy of D that the FP32 LU factors.
// Splitting the pair evaluation keeps each kernel's registers and code small
// enough for several CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int ASM_ROWS = 128;
constexpr int ASM_TJ = 32;
#ifndef ASM_MINB_RANKINE
#define ASM_MINB_RANKINE 3
#endif
// CTAs per SM of the wave pass (128 and 102 registers at most): measured on the barge
// step, the finite-depth pass is fastest at 4 (at 5 its spills double and the
// assembly takes 1.8 ms more); the deep-water pass spills the same at 96
// registers as at 128 (its stack holds local arrays), and 5 CTAs save about
// 0.5 ms of the step's assembly
#ifndef ASM_MINB_WAVE_FD
#define ASM_MINB_WAVE_FD 4
#endif
#ifndef ASM_MINB_WAVE_INFD
#define ASM_MINB_WAVE_INFD 5
#endif

struct AsmOut {
  double2* d;           // D+ (and D-) of frequency slot s at d + s * slot_stride
  double2* s;           // S+ (and S-) likewise
  long long slot_stride;
  float2* d32 = nullptr;   // optional FP32 copy of the final D (same layout), for the mixed LU
  const double2* rk = nullptr;   // Rankine cache of the launch's depth regime (null: read the real parts)
};

// Ragged batches (frequency slots of different bodies in one launch): the
// mesh and output place of each slot. Without it every slot uses the
// kernel's own mesh arguments and slot * slot_stride.
struct SlotMesh {
  const PanelRec* rec;
  const double* rows;
  long long off;   // element offset of the slot's D+ (and S+, FP32 copy); D-/S- follow after n*n
  int n;
  int nsymy;
  double zer;
  const double2* rk;   // the body's Rankine cache for the slot's depth regime, or null
};

__device__ __forceinline__ void stage_panels(const PanelRec* __restrict__ rec, int j0, int nj, PanelRec* sp) {
  const double* src = reinterpret_cast<const double*>(rec + j0);
  double* dst = reinterpret_cast<double*>(sp);
  const int nw = nj * (int)(sizeof(PanelRec) / 8);
  for (int i = threadIdx.x; i < nw; i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ void stage_params(const OmegaParams* __restrict__ om, OmegaParams* som) {
  const double* src = reinterpret_cast<const double*>(om);
  double* dst = reinterpret_cast<double*>(som);
  for (int i = threadIdx.x; i < (int)(sizeof(OmegaParams) / 8); i += blockDim.x) dst[i] = src[i];
}

template <bool FD>
__global__ void __launch_bounds__(ASM_ROWS, ASM_MINB_RANKINE) rankine_kernel(GreenCtx g, const OmegaParams* __restrict__ oms,
                                                           const int* __restrict__ slots,
                                                           const PanelRec* __restrict__ rec,
                                                           const double* __restrict__ rows, int N, AsmOut out,
                                                           const SlotMesh* __restrict__ meshes) {
  __shared__ PanelRec sp[ASM_TJ];
  __shared__ OmegaParams som;
  const int slot = slots[blockIdx.z];
  long long base = slot * out.slot_stride;
  if (meshes) {
    const SlotMesh m = meshes[slot];
    rec = m.rec;
    rows = m.rows;
    N = m.n;
    g.nsymy = m.nsymy;
    g.zer = m.zer;
    base = m.off;
    if (m.rk) return;   // the wave pass reads this slot's Rankine part from its cache (whole CTA)
  }
  const int j0 = blockIdx.y * ASM_TJ;
  if (j0 >= N || (int)blockIdx.x * ASM_ROWS >= N) return;   // beyond a smaller slot's order (whole CTA)
  stage_params(oms + slot, &som);
  const int nj = min(ASM_TJ, N - j0);
  stage_panels(rec, j0, nj, sp);
  __syncthreads();
  const int I = blockIdx.x * ASM_ROWS + threadIdx.x;
  if (I >= N) return;
  const double XGI = rows[I], YGI = rows[N + I], ZGI = rows[2 * N + I];
  const double XNI = rows[3 * N + I], YNI = rows[4 * N + I], ZNI = rows[5 * N + I];
  const long long NN = (long long)N * N;
  double2* od = out.d + base;
  double2* os = out.s + base;
#pragma unroll 1
  for (int jj = 0; jj < nj; ++jj) {
    const int J = j0 + jj;
    RealOut r;
    pair_rankine<FD>(g, som, som.ambda, som.ar, XGI, YGI, ZGI, XNI, YNI, ZNI, I == J, sp[jj], r);
    const long long q = I + (long long)N * J;
    od[q] = make_double2(r.dp, 0.);
    os[q] = make_double2(r.sp, 0.);
    if (g.nsymy == 1) {
      od[NN + q] = make_double2(r.dm, 0.);
      os[NN + q] = make_double2(r.sm, 0.);
    }
  }
}

// Rankine part of every pair of one mesh into its cache: rk[I + N J] =
// (D+, S+) real parts, rk[N N + I + N J] = (D-, S-) when nsymy = 1. DH is
// twice the depth in finite depth (seabed image), 0 in deep water.
template <bool FD>
__global__ void __launch_bounds__(ASM_ROWS, ASM_MINB_RANKINE) rankine_cache_kernel(GreenCtx g, double DH,
                                                                 const PanelRec* __restrict__ rec,
                                                                 const double* __restrict__ rows, int N,
                                                                 double2* __restrict__ rk) {
  __shared__ PanelRec sp[ASM_TJ];
  const int j0 = blockIdx.y * ASM_TJ;
  const int nj = min(ASM_TJ, N - j0);
  stage_panels(rec, j0, nj, sp);
  __syncthreads();
  const int I = blockIdx.x * ASM_ROWS + threadIdx.x;
  if (I >= N) return;
  const double XGI = rows[I], YGI = rows[N + I], ZGI = rows[2 * N + I];
  const double XNI = rows[3 * N + I], YNI = rows[4 * N + I], ZNI = rows[5 * N + I];
  const long long NN = (long long)N * N;
#pragma unroll 1
  for (int jj = 0; jj < nj; ++jj) {
    const int J = j0 + jj;
    RankineOut r;
    rankine<FD>(g, DH, XGI, YGI, ZGI, I == J, sp[jj], r);
    const long long q = I + (long long)N * J;
    rk[q] = make_double2(r.VSXP * XNI + r.VSYP * YNI + r.VSZP * ZNI, r.FSP);
    if (g.nsymy == 1) rk[NN + q] = make_double2(r.VSXM * XNI + r.VSYM * YNI + r.VSZM * ZNI, r.FSM);
  }
}

// ---------------------------------------------------------------------------
// Wave pass over the upper triangle of 16 x 16 tiles: a pair of submerged
// panels is evaluated once for both orders (finite depth: wave_fd_sym and the
// exponential images of the same branch, fd_images_pair; deep water:
// wave_infd_both), any other pair once per order (pair_wave); both the tile
// and its transpose are added to the real parts and written to the imaginary
// parts, the tile straight from the evaluating threads, its transpose column
// by column through shared memory.
// ---------------------------------------------------------------------------
constexpr int WS_T = 16;
constexpr int WS_THREADS = 128;

// linear index t over the upper triangle (a <= b) of a T x T tile grid
NB_HD __forceinline__ void tri_tile(int t, int T, int& a, int& b) {
  auto start = [T](int r) { return r * T - r * (r - 1) / 2; };
  const double q = 2. * T + 1.;
  int r = (int)((q - sqrt(q * q - 8. * t)) * 0.5);
  r = max(0, min(T - 1, r));
  while (r > 0 && start(r) > t) --r;
  while (r < T - 1 && start(r + 1) <= t) ++r;
  a = r;
  b = r + (t - start(r));
}

// Exponential images (VNSFD, COMPUTE_GREEN_FD.f90:635-706) of both orders of
// a pair of submerged panels, added to the real parts of D+/-, S+/-.
NB_HD __forceinline__ void fd_images_pair(const GreenCtx& g, const OmegaParams& om, const PanelRec& PI,
                                               const PanelRec& PJ, int NJJ, bool both, PairOut& oij, PairOut& oji) {
  ImageSums S;
  fd_image_sums(g, om.h, om.ambda, om.ar, om.nexp + 1, PI.xg, PI.yg, PI.zg, PJ.xg, PJ.yg, PJ.zg, NJJ, S);
  const double QPI = 4. * 3.141592653589793;
#pragma unroll
  for (int order = 0; order < 2; ++order) {
    if (order == 1 && !both) break;
    const bool tr = order == 1;
    const PanelRec& C = tr ? PJ : PI;   // collocation panel
    const double act = -0.5 * (tr ? PI.aire : PJ.aire) / QPI;
    double fs[2], vx[2], vy[2], vz[2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      fs[b] = act * S.fs[b];
      const double dx = tr ? -S.dx[b] : S.dx[b];
      const double dy = (tr && b == 0) ? -S.dy[b] : S.dy[b];
      vx[b] = -dx * (act * S.sa[b]);
      vy[b] = -dy * (act * S.sa[b]);
      vz[b] = tr ? act * S.m2[b] : -(act * S.m1[b]);
    }
    PairOut& o = tr ? oji : oij;
    if (NJJ == 2) {
      o.dp_re += (vx[0] + vx[1]) * C.xn + (vy[0] + vy[1]) * C.yn + (vz[0] + vz[1]) * C.zn;
      o.dm_re += (vx[0] - vx[1]) * C.xn + (vy[0] - vy[1]) * C.yn + (vz[0] - vz[1]) * C.zn;
      o.sp_re += fs[0] + fs[1];
      o.sm_re += fs[0] - fs[1];
    } else {
      const double d = vx[0] * C.xn + vy[0] * C.yn + vz[0] * C.zn;
      o.dp_re += d;
      o.dm_re += d;
      o.sp_re += fs[0];
      o.sm_re += fs[0];
    }
  }
}

// one order of a pair with a panel at the free surface (rare; kept out of line)
template <bool FD>
NB_HD __noinline__ void pair_wave_ordered(const GreenCtx& g, const OmegaParams& om, const PanelRec& PC,
                                               const PanelRec& PS, PairOut& out) {
  pair_wave<FD>(g, om, PC.xg, PC.yg, PC.zg, PC.xn, PC.yn, PC.zn, PS, out);
}

// Deep water (VNSINFD, one image at ZI + ZJ): every sum is the same for both
// orders except the horizontal gradient, whose x part and direct-reflection y
// part change sign.
NB_HD __forceinline__ void wave_infd_both(const GreenCtx& g, const OmegaParams& om, const PanelRec& PI,
                                               const PanelRec& PJ, int NJJ, bool both, PairOut& oij, PairOut& oji) {
  WaveJJ w[2];
  wave_infd_pair(g, om, PI.xg, PI.yg, PI.zg, PJ, NJJ, w);
  if (NJJ == 1) w[1] = WaveJJ{0, 0, 0, 0, 0, 0, 0, 0};
  wave_combine<false>(om, PJ.aire, NJJ, w, PI.xn, PI.yn, PI.zn, oij);
  if (!both) return;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    w[b].VSX1 = -w[b].VSX1;
    w[b].VSX2 = -w[b].VSX2;
    if (b == 0) {
      w[b].VSY1 = -w[b].VSY1;
      w[b].VSY2 = -w[b].VSY2;
    }
  }
  wave_combine<false>(om, PI.aire, NJJ, w, PJ.xn, PJ.yn, PJ.zn, oji);
}

// Transposed results of a tile, one array per PairOut field, rows padded to
// T + 1 so that both the store (thread = row i) and the load (thread = column
// j) touch distinct banks.
struct TileT {
  double v[8][WS_T * (WS_T + 1)];
  NB_HD __forceinline__ void put(int i, int j, const PairOut& r) {
    const int o = i * (WS_T + 1) + j;
    v[0][o] = r.dp_re; v[1][o] = r.dp_im; v[2][o] = r.dm_re; v[3][o] = r.dm_im;
    v[4][o] = r.sp_re; v[5][o] = r.sp_im; v[6][o] = r.sm_re; v[7][o] = r.sm_im;
  }
  NB_HD __forceinline__ PairOut get(int i, int j) const {
    const int o = i * (WS_T + 1) + j;
    return PairOut{v[0][o], v[1][o], v[2][o], v[3][o], v[4][o], v[5][o], v[6][o], v[7][o]};
  }
};

template <bool FD>
__global__ void __launch_bounds__(WS_THREADS, FD ? ASM_MINB_WAVE_FD : ASM_MINB_WAVE_INFD) wave_sym_kernel(
    GreenCtx g, const OmegaParams* __restrict__ oms, const int* __restrict__ slots, const PanelRec* __restrict__ rec,
    int N, AsmOut out, const SlotMesh* __restrict__ meshes) {
  // (A_i, B_j) goes out from the thread that evaluates it (consecutive
  // threads hold consecutive rows i); (B_j, A_i) is staged here and written
  // after the tile, row j by consecutive threads. Keeping only the transposed
  // half in shared memory leaves more of the SM's L1 to the table gathers.
  __shared__ TileT res;
  __shared__ PanelRec pa[WS_T], pb[WS_T];
  __shared__ OmegaParams som;
  const int slot = slots[blockIdx.z];
  long long base = slot * out.slot_stride;
  const double2* rk = out.rk;
  if (meshes) {
    const SlotMesh m = meshes[slot];
    rec = m.rec;
    N = m.n;
    g.nsymy = m.nsymy;
    g.zer = m.zer;
    base = m.off;
    rk = m.rk;
  }
  const int T = (N + WS_T - 1) / WS_T;
  if ((int)blockIdx.x >= T * (T + 1) / 2) return;   // beyond a smaller slot's tiles (whole CTA)
  int ta, tb;
  tri_tile(blockIdx.x, T, ta, tb);
  stage_params(oms + slot, &som);
  const int a0 = ta * WS_T, b0 = tb * WS_T;
  const int na = min(WS_T, N - a0), nb = min(WS_T, N - b0);
  stage_panels(rec, a0, na, pa);
  stage_panels(rec, b0, nb, pb);
  __syncthreads();
  const bool diag = ta == tb;
  const int NJJ = g.nsymy + 1;
  const long long NN = (long long)N * N;
  double2* od = out.d + base;
  double2* os = out.s + base;
  float2* o32 = out.d32 ? out.d32 + base : nullptr;
  // Rankine real parts of entry o (within the slot) of the plus and minus classes
  auto rankine_at = [&](long long o, int cls) {
    if (rk) return rk[cls * NN + o];
    return make_double2(od[cls * NN + o].x, os[cls * NN + o].x);
  };
  auto add = [&](long long o, const PairOut& r) {
    double2 rr = rankine_at(o, 0);
    const double2 dn = make_double2(rr.x + r.dp_re, r.dp_im);
    od[o] = dn;
    os[o] = make_double2(rr.y + r.sp_re, r.sp_im);
    if (o32) o32[o] = make_float2((float)dn.x, (float)dn.y);
    if (NJJ == 2) {
      rr = rankine_at(o, 1);
      const double2 dm = make_double2(rr.x + r.dm_re, r.dm_im);
      od[NN + o] = dm;
      os[NN + o] = make_double2(rr.y + r.sm_re, r.sm_im);
      if (o32) o32[NN + o] = make_float2((float)dm.x, (float)dm.y);
    }
  };
  auto live = [&](int i, int j) { return i < na && j < nb && !(diag && i > j); };
#pragma unroll 1
  for (int q = threadIdx.x; q < WS_T * WS_T; q += WS_THREADS) {
    const int i = q % WS_T, j = q / WS_T;
    const bool lv = live(i, j);
    const PanelRec& PI = pa[i];
    const PanelRec& PJ = pb[j];
    const bool both = !(diag && i == j);
    PairOut oij, oji;
    if (!lv) {
    } else if (PI.zg < g.zer && PJ.zg < g.zer) {
      if (FD) {
        if (!wave_fd_sym(g, som, PI, PJ, NJJ, both, oij, oji)) {
          set_status(g.status, ST_AKZ_UNDEFINED);
          oij = oji = PairOut{0, 0, 0, 0, 0, 0, 0, 0};
        }
        fd_images_pair(g, som, PI, PJ, NJJ, both, oij, oji);
      } else {
        wave_infd_both(g, som, PI, PJ, NJJ, both, oij, oji);
      }
    } else {
      pair_wave_ordered<FD>(g, som, PI, PJ, oij);
      if (both) pair_wave_ordered<FD>(g, som, PJ, PI, oji);
    }
    // the warp stores its rows together: each column segment goes out whole
    __syncwarp();
    if (!lv) continue;
    add((a0 + i) + (long long)N * (b0 + j), oij);
    if (both) res.put(i, j, oji);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < WS_T * WS_T; q += WS_THREADS) {
    // entry (b0 + j, a0 + i); the diagonal of a diagonal tile went out above
    const int j = q % WS_T, i = q / WS_T;
    if (live(i, j) && !(diag && i == j)) add((b0 + j) + (long long)N * (a0 + i), res.get(i, j));
  }
}

}  // namespace nb200
