// Pre-processor on the device: the right-hand sides and integration normals
// that the reference pre-processor writes to Normalvelocities.dat,
// Integration.dat and FKForce.dat (preProcessor/Main.f90:201-243).
//   panel quantities   preProcessor/Mesh.f90:197-222 (two-triangle centroid,
//                      normal of the summed cross products, area)
//   incident wave      Common/Environment.f90:86-100 (Compute_Wave: pressure
//                      and velocity of the linear incident wave, CIH/SIH)
//   body conditions    preProcessor/BodyConditions.f90:27-137 (diffraction
//                      -v_I . n, radiation n . d or n . (d x (x - axis)))
//   integration        preProcessor/Integration.f90:27-86 (NDS = area x the
//                      radiation vector of each force case)
//   Froude-Krylov      preProcessor/Main.f90:223-235 (-sum NDS p_I)
// One thread per panel and mesh half (the y-mirror of a symmetric mesh).
#pragma once
#include "common.cuh"

namespace nb200 {

struct PreDof {
  int kind;            // 1 translation along dir, 2 rotation about the axis through `axis`
  int body;            // panels of this body only (1-based)
  double dir[3], axis[3];
};

struct PreWave {
  double w, k, cb, sb;   // frequency, pre-processor wave number, cos/sin of the heading
};

NB_HD __forceinline__ void pre_panel(const double* __restrict__ xyz, const int* __restrict__ m, int i, double* xm,
                                     double* nrm, double& area) {
  double x[4][3];
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int c = 0; c < 3; ++c) x[l][c] = xyz[3 * (m[4 * i + l] - 1) + c];
  double u1[3], v1[3], u2[3], v2[3], w1[3], w2[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    u1[c] = x[1][c] - x[0][c];
    v1[c] = x[3][c] - x[1][c];
    u2[c] = x[3][c] - x[2][c];
    v2[c] = x[1][c] - x[2][c];
  }
  w1[0] = u1[1] * v1[2] - u1[2] * v1[1];
  w1[1] = u1[2] * v1[0] - u1[0] * v1[2];
  w1[2] = u1[0] * v1[1] - u1[1] * v1[0];
  w2[0] = u2[1] * v2[2] - u2[2] * v2[1];
  w2[1] = u2[2] * v2[0] - u2[0] * v2[2];
  w2[2] = u2[0] * v2[1] - u2[1] * v2[0];
  const double a1 = 0.5 * sqrt(w1[0] * w1[0] + w1[1] * w1[1] + w1[2] * w1[2]);
  const double a2 = 0.5 * sqrt(w2[0] * w2[0] + w2[1] * w2[1] + w2[2] * w2[2]);
  area = a1 + a2;
  const double un[3] = {w1[0] + w2[0], w1[1] + w2[1], w1[2] + w2[2]};
  const double nn = sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    xm[c] = (1. / 3) * (x[0][c] + x[1][c] + x[3][c]) * (a1 / area) + (1. / 3) * (x[1][c] + x[2][c] + x[3][c]) * (a2 / area);
    nrm[c] = un[c] / nn;
  }
}

// radiation velocity . normal for one DOF at (x, n)
NB_HD __forceinline__ double pre_dof(const PreDof& d, const double* x, const double* n) {
  if (d.kind == 1) return n[0] * d.dir[0] + n[1] * d.dir[1] + n[2] * d.dir[2];
  const double r0 = x[0] - d.axis[0], r1 = x[1] - d.axis[1], r2 = x[2] - d.axis[2];
  const double v0 = d.dir[1] * r2 - d.dir[2] * r1, v1 = d.dir[2] * r0 - d.dir[0] * r2, v2 = d.dir[0] * r1 - d.dir[1] * r0;
  return n[0] * v0 + n[1] * v1 + n[2] * v2;
}

// diffraction condition -v_I . n of the incident wave pw at (xm, n), with the
// depth factors CIH/SIH that the Froude-Krylov pressure also needs
NB_HD __forceinline__ void pre_diffraction(const PreWave& pw, double g, double depth, double xeff, double yeff,
                                           const double* xm, const double* n, double& vr, double& vi, double& cih,
                                           double& ce, double& se) {
  const double k = pw.k, kh = k * depth;
  double sih;
  if (kh <= 20. && kh > 0.) {
    cih = cosh(k * (xm[2] + depth)) / cosh(kh);
    sih = sinh(k * (xm[2] + depth)) / cosh(kh);
  } else {
    cih = sih = exp(k * xm[2]);
  }
  const double wbar = (xm[0] - xeff) * pw.cb + (xm[1] - yeff) * pw.sb;
  sincos(k * wbar, &se, &ce);
  const double gwk = g / pw.w * k;
  // v = (gwk cb cih e, gwk sb cih e, -i gwk sih e), e = exp(i k wbar)
  const double vxr = gwk * pw.cb * cih * ce, vxi = gwk * pw.cb * cih * se;
  const double vyr = gwk * pw.sb * cih * ce, vyi = gwk * pw.sb * cih * se;
  const double vzr = gwk * sih * se, vzi = -gwk * sih * ce;
  vr = -(vxr * n[0] + vyr * n[1] + vzr * n[2]);
  vi = -(vxi * n[0] + vyi * n[1] + vzi * n[2]);
}

// nvel: per frequency w, (nbeta + ndof) columns of 2^s N complex (headings
// then DOFs, the pre-processor's problem order); nds: nforce x 2^s N;
// fk: nforce x nbeta x nomega complex, accumulated with atomics (zeroed first).
__global__ void __launch_bounds__(128)
    preproc_kernel(const double* __restrict__ xyz, const int* __restrict__ m1234, const int* __restrict__ pbody, int nfa,
                   int nsymy, double rho, double g, double depth, double xeff, double yeff,
                   const PreWave* __restrict__ waves, int nomega, int nbeta, const PreDof* __restrict__ dofs, int ndof,
                   const PreDof* __restrict__ forces, int nforce, double2* __restrict__ nvel, double* __restrict__ nds,
                   double2* __restrict__ fk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int half = blockIdx.y;
  if (i >= nfa || half > nsymy) return;
  double xm[3], n[3], area;
  pre_panel(xyz, m1234, i, xm, n, area);
  if (half) {
    xm[1] = -xm[1];
    n[1] = -n[1];
  }
  const int body = pbody ? pbody[i] : 1;
  const int nc = nfa * (nsymy + 1), row = i + half * nfa, npb = nbeta + ndof;
  for (int q = 0; q < nforce; ++q)
    if (nds) nds[q + (long long)nforce * row] = forces[q].body == body ? pre_dof(forces[q], xm, n) * area : 0.;
  for (int w = 0; w < nomega; ++w) {
    for (int d = 0; d < ndof; ++d) {
      const double v = dofs[d].body == body ? pre_dof(dofs[d], xm, n) : 0.;
      nvel[row + (long long)nc * (nbeta + d + (long long)npb * w)] = make_double2(v, 0.);
    }
    for (int b = 0; b < nbeta; ++b) {
      const PreWave& pw = waves[w * nbeta + b];
      double vr, vi, cih, ce, se;
      pre_diffraction(pw, g, depth, xeff, yeff, xm, n, vr, vi, cih, ce, se);
      nvel[row + (long long)nc * (b + (long long)npb * w)] = make_double2(vr, vi);
      if (fk) {
        const double pr = rho * g * cih * ce, pi = rho * g * cih * se;
        for (int q = 0; q < nforce; ++q) {
          const double a = forces[q].body == body ? pre_dof(forces[q], xm, n) * area : 0.;
          double2* f = fk + q + (long long)nforce * (b + (long long)nbeta * w);
          atomicAdd(&f->x, -a * pr);
          atomicAdd(&f->y, -a * pi);
        }
      }
    }
  }
}

// Right-hand sides of serving requests: request r is (resident body, omega,
// heading) with the body's ndof radiation DOFs; its NVEL block (2^s N) x
// (1 + ndof) at nvel + nvel_off holds the diffraction column at the heading,
// then the radiation columns, as the pre-processor orders the problems of one
// frequency (one thread per panel and mesh half; grid.z = request).
struct ReqDesc {
  const double* xyz;
  const int* m1234;
  const PreDof* dofs;
  PreWave wave;
  double g, depth;
  long long nvel_off;
  int nfa, nsymy, ndof;
};

__global__ void __launch_bounds__(128) request_rhs_kernel(const ReqDesc* __restrict__ reqs, double2* __restrict__ nvel) {
  const ReqDesc rq = reqs[blockIdx.z];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int half = blockIdx.y;
  if (i >= rq.nfa || half > rq.nsymy) return;
  double xm[3], n[3], area;
  pre_panel(rq.xyz, rq.m1234, i, xm, n, area);
  if (half) {
    xm[1] = -xm[1];
    n[1] = -n[1];
  }
  const int nc = rq.nfa * (rq.nsymy + 1), row = i + half * rq.nfa;
  double2* out = nvel + rq.nvel_off;
  double vr, vi, cih, ce, se;
  pre_diffraction(rq.wave, rq.g, rq.depth, 0., 0., xm, n, vr, vi, cih, ce, se);
  out[row] = make_double2(vr, vi);
  for (int d = 0; d < rq.ndof; ++d) out[row + (long long)nc * (1 + d)] = make_double2(pre_dof(rq.dofs[d], xm, n), 0.);
}

}  // namespace nb200
