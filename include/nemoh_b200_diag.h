/*
 * nemoh_b200 diagnostics: the host-side scalar setup of one frequency,
 * exported so that it can be checked against an independent restatement of
 * the reference routines without a GPU. Not needed to run a solve.
 */
#ifndef NEMOH_B200_DIAG_H
#define NEMOH_B200_DIAG_H
#ifdef __cplusplus
extern "C" {
#endif

/* X0: root of x tanh x = ak (Solver/Core/COMPUTE_GREEN_FD.f90:1635-1680) */
int nemoh_b200_diag_dispersion_root(double ak, double* root);
/* LISC: finite-depth exponential fit (COMPUTE_GREEN_FD.f90:1007-1077);
 * ambda[31], ar[31] receive AMBDA(1..31), AR(1..31) */
int nemoh_b200_diag_exponential_fit(double akh, double amh, int* nexp, double* ambda, double* ar);
/* CINT_INFD / CINT_FD: returns the node count; qq, cq hold >= 101 entries */
int nemoh_b200_diag_theta_quadrature(double akk, double* qq, double* cq);
/* thresholds of the table-stencil indices, 48 each: for every index k the
 * smallest x whose truncated log10 formula gives >= k, found by bisection on the
 * double bit pattern with the host's log10 */
int nemoh_b200_diag_stencil_thresholds(double* kj8, double* kj5, double* ki5);
/* autotuner of the triangular sweep: keys tuned in this process so far, and
 * the sweep chosen for a batch of nsys systems of order n with nrhs
 * right-hand sides in single (1) or double (0) precision: the cluster size
 * (1, 2, 4, 8) of the cluster sweep, 16 for the dataflow sweep, 0 if not
 * tuned */
int nemoh_b200_diag_sweep_tuning(long long* keys_tuned, int n, int nsys, int nrhs, int single, int* cluster_size);
/* measured FP64 FMA throughput of a device (TFLOP/s, 2 FLOP per FMA): the
 * best of four launches of independent FMA chains on every SM */
int nemoh_b200_diag_fp64_peak(int device, double* tflops);
/* bounded-wait check of the dataflow sweep: a launch whose only item waits on
 * a ready flag that nothing raises; returns the status word the kernel left
 * (31 = the wait ran out) and the launch's duration */
int nemoh_b200_diag_sweep_timeout(int device, int* status, double* ms);

#ifdef __cplusplus
}
#endif
#endif
