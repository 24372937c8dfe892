// Host-side scalar setup of the per-frequency solve (see fd_setup.cpp).
#pragma once
#include "common.cuh"

namespace nb200 {

// X0: root m0*h of x*tanh(x) = ak, bisection to 5e-6 (COMPUTE_GREEN_FD.f90:1635-1680)
int finite_depth_root(double ak, double* out);

// Pre-processor wave number (Common/Environment.f90:45-85): bisection to 1e-6
// on x tanh x = w^2 h / g; w^2 / g in deep water or for w^2 h / g > 20.
double preproc_wavenumber(double w, double g, double depth);

// LISC: fit of the finite-depth kernel by exponentials; ambda/ar are 1-based,
// size MAX_NEXP+1 (COMPUTE_GREEN_FD.f90:1007-1077)
int exponential_fit(double akh, double amh, int* nexp, double* ambda, double* ar);

// CINT_INFD / CINT_FD: theta nodes qq[1..n], weights cq[1..n]; returns n
int theta_quadrature(double akk, double* qq, double* cq);

// CREK nodes: xr[1..328], xz[1..46]
void table_nodes(double* xr, double* xz);

// COFINT: 251-point Simpson nodes/weights (1-based)
void simpson_251(double* cqt, double* qqt);

// thresholds that make the device's table-stencil indices exact
void stencil_thresholds(StencilThresholds* t);

}  // namespace nb200
