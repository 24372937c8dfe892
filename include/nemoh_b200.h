/*
 * nemoh_b200 C-ABI: the per-frequency BEM solve of Nemoh on an NVIDIA B200.
 *
 * Drop-in for the reference Solver's direct BEM solve:
 *   SOLVE_POTENTIAL_INFD_DIRECT(NVEL)          Solver/Core/SOLVE_BEM_INFD_DIRECT.f90:34
 *   SOLVE_POTENTIAL_FD_DIRECT(NVEL,AMH,NEXP)   Solver/Core/SOLVE_BEM_FD_DIRECT.f90:33
 * as dispatched by SOLVE_BVP (Solver/Core/SOLVE_BEM.f90:28-117), with the mesh
 * and environment set up as INITIALIZE does (Solver/Core/INITIALIZATION.f90:28-69).
 *
 * Conventions
 *  - Arrays are caller-owned host buffers unless a name ends in _device.
 *  - Complex numbers are interleaved (re, im) doubles; matrices column-major.
 *  - Every call returns a status: 0 = OK, otherwise one of NEMOH_B200_E*;
 *    nemoh_b200_last_error() gives the message. Each STOP of the reference
 *    maps to a status (no process exit).
 *  - A context is used by one host thread at a time. Separate contexts may
 *    run concurrently on separate host threads.
 */
#ifndef NEMOH_B200_H
#define NEMOH_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nemoh_ctx nemoh_ctx;

/* status codes */
#define NEMOH_B200_OK 0
#define NEMOH_B200_EINVAL 1          /* bad argument */
#define NEMOH_B200_EPANEL_AREA 2     /* PREPARE_MESH.f90:112-120 "area of panel is too small" */
#define NEMOH_B200_EPIVOT 3          /* M_SOLVER.f90:49-52,61-64 "PIVOT INFERIEUR A 1e-20" */
#define NEMOH_B200_EOMEGA 4          /* COMPUTE_GREEN_INFD.f90:252-255 |W| < 1e-4 */
#define NEMOH_B200_ELISC 5           /* COMPUTE_GREEN_FD.f90:1073 positive exponent */
#define NEMOH_B200_ESPRBM 6          /* COMPUTE_GREEN_FD.f90:1311-1314 root finder failure */
#define NEMOH_B200_EDISPERSION 7     /* COMPUTE_GREEN_FD.f90:1656-1660 no dispersion root */
#define NEMOH_B200_EAKZ 8            /* COMPUTE_GREEN_INFD.f90:284-289 wave term undefined */
#define NEMOH_B200_EIO 9             /* file format / IO (drop-in driver) */
#define NEMOH_B200_EHOUSRS 10        /* COMPUTE_GREEN_FD.f90:1461-1477 least squares */
#define NEMOH_B200_ECUDA 20          /* CUDA runtime error */
#define NEMOH_B200_ENOMEM 21         /* device memory exhausted / admission refused */
#define NEMOH_B200_ENODEV 22         /* no CUDA device */
#define NEMOH_B200_ECAPACITY 23      /* size beyond a documented limit */
#define NEMOH_B200_ETIMEOUT 30       /* a bounded device-side wait gave up */

/* precision modes */
#define NEMOH_B200_FP64 0            /* FP64 assembly, FP64 LU */
#define NEMOH_B200_MIXED 1           /* FP64 assembly, FP32 LU with split-BF16 tensor-core updates,
                                        FP64 iterative refinement */

/* Create a context on a CUDA device; builds the Green-function tables
 * (CREK, Solver/NEMOH.f90:179-274) on that device. */
int nemoh_b200_create(nemoh_ctx** ctx, int device, int precision_mode);
int nemoh_b200_destroy(nemoh_ctx* ctx);
const char* nemoh_b200_last_error(const nemoh_ctx* ctx);

/* Mesh and environment: INITIALIZE + PRE_PROC_MESH (INITIALIZATION.f90:44-67,
 * PREPARE_MESH.f90:30-180). xyz is 3 x np (x,y,z per node); m1234 is
 * 4 x nfa 1-based node ids; nsymy = 1 for a y-symmetric half mesh.
 * depth = 0 means infinite depth. Resets the factor cache. */
int nemoh_b200_set_mesh(nemoh_ctx* ctx, int np, int nfa, int nsymy, const double* xyz, const int* m1234,
                        double rho, double g, double depth);

/* One problem, the reference's boundary exactly (SOLVE_BEM.f90:62-96 with
 * SOLVE_POTENTIAL_*_DIRECT): period T, normal velocities nvel (2^nsymy * nfa
 * complex). Outputs (nfa complex each, any may be NULL): source strengths
 * zigb, zigs and boundary potentials zpb, zps; nexp (finite depth exponential
 * count, 0 in deep water). The factorization is cached while 2*pi/T equals
 * the previous call's (the reference's w_previous, SOLVE_BEM_INFD_DIRECT.f90:82). */
int nemoh_b200_solve_problem(nemoh_ctx* ctx, double period, const double* nvel, double* zigb, double* zigs,
                             double* zpb, double* zps, int* nexp);

/* Batched fast path: nomega frequencies, each with nrhs problems (1 <= nrhs <= 16;
 * NEMOH_B200_EINVAL below, NEMOH_B200_ECAPACITY above, both before any copy).
 * nvel: (2^s nfa) x nrhs x nomega complex; nds: nint x (2^s nfa) real
 * (mesh/Integration.dat, NEMOH.f90:88-94); force: nint x nrhs x nomega
 * complex, Force = -sum_c PRESSURE(c) NDS(i,c) with PRESSURE = rho i W phi
 * (NEMOH.f90:137-141, SOLVE_BEM.f90:91-96). Frequencies are processed in the
 * given order (the order matters only for the reference's free-surface-panel
 * quadrature state: in deep water the theta sum runs over the node count NQ
 * left by the last finite-depth frequency, SOLVE_BEM_INFD_DIRECT.f90:79). */
int nemoh_b200_solve_frequencies(nemoh_ctx* ctx, int nomega, const double* omegas, int nrhs, const double* nvel,
                                 int nint, const double* nds, double* force);

/* Same with device-resident inputs/outputs (pointers from cudaMalloc on the
 * context's device) on the given CUDA stream (cudaStream_t as void*). */
int nemoh_b200_solve_frequencies_device(nemoh_ctx* ctx, int nomega, const double* omegas, int nrhs,
                                        const double* nvel_device, int nint, const double* nds_device,
                                        double* force_device, void* stream);

/* Kochin function (COMPUTE_KOCHIN.f90:25-152, as called by SOLVE_BEM.f90:98-102):
 * for source strengths zigb, zigs (nfa x nprob complex each, as returned by
 * nemoh_b200_solve_problem; zigs unused without symmetry) of problems at period
 * `period`, H(theta) at the ntheta directions theta (radians, mesh/Kochin.dat)
 * about the wave measurement point (xeff, yeff) of Nemoh.cal (yeff is taken
 * as 0 on symmetric meshes, INITIALIZATION.f90:60). hkochin: ntheta x nprob
 * complex (theta fastest). */
int nemoh_b200_kochin(nemoh_ctx* ctx, double period, double xeff, double yeff, int ntheta, const double* theta,
                      int nprob, const double* zigb, const double* zigs, double* hkochin);

/* Free-surface elevation (COMPUTE_POTENTIAL_DOMAIN.f90:24-82 with
 * COMPUTE_GREEN_FREESURFACE.f90, as called at SOLVE_BEM.f90:104-109): for source
 * strengths zigb, zigs (nfa x nprob complex each; zigs unused without symmetry)
 * of problems at period `period`, ETA = i W / G PHI at the npts points
 * (x, y, 0) of xy (2 x npts, mesh/Freesurface.dat). eta: npts x nprob complex. */
int nemoh_b200_free_surface(nemoh_ctx* ctx, double period, int npts, const double* xy, int nprob,
                            const double* zigb, const double* zigs, double* eta);

/* Radiation impulse response functions of the post-processor (Compute_IRF,
 * postProcessor/IRF.f90:100-127): from damping and added mass (nw x nrad x
 * nint, w fastest; w nonzero) the kernels K at t_i = i dt, i < ntime (ntime x
 * nrad x nint, time fastest) by the trapezoid rule over w, and the
 * infinite-frequency added mass ainf (nrad x nint) estimated from K. Needs a
 * context (for its device and stream), not a mesh. */
int nemoh_b200_irf(nemoh_ctx* ctx, int nw, const double* w, int nrad, int nint, const double* damping,
                   const double* added_mass, int ntime, double dt, double* K, double* ainf);

/* Pre-processor body conditions on the device for the current mesh
 * (preProcessor/Main.f90:201-243 with Mesh.f90:197-222, BodyConditions.f90:27-137,
 * Environment.f90:45-100, Integration.f90:27-86): for nomega frequencies, nbeta
 * headings (radians) and ndof radiation DOFs (kind 1 translation along dir, 2
 * rotation about the axis through `axis` with direction dir; 3 doubles each;
 * dof_body / panel_body select the panels of a body, both may be NULL for one
 * body) it writes
 *   nvel  (2^s nfa) x (nbeta + ndof) x nomega complex: NVEL of Normalvelocities.dat
 *         (per frequency the headings, then the DOFs);
 *   nds   nforce x (2^s nfa): the generalised normals of Integration.dat (or NULL);
 *   fk    nforce x nbeta x nomega complex: Froude-Krylov forces (or NULL),
 * with the wave measurement point (xeff, yeff) and the mesh's rho, g, depth. */
int nemoh_b200_body_conditions(nemoh_ctx* ctx, const int* panel_body, double xeff, double yeff, int nomega,
                               const double* omegas, int nbeta, const double* betas, int ndof, const int* dof_kind,
                               const int* dof_body, const double* dof_dir, const double* dof_axis, int nforce,
                               const int* force_kind, const int* force_body, const double* force_dir,
                               const double* force_axis, double* nvel, double* nds, double* fk);
/* Same with the outputs in device memory of the context's device, ordered
 * after the work already on `stream` (cudaStream_t) and before what follows;
 * nvel_device can go straight to nemoh_b200_solve_frequencies_device. */
int nemoh_b200_body_conditions_device(nemoh_ctx* ctx, const int* panel_body, double xeff, double yeff, int nomega,
                                      const double* omegas, int nbeta, const double* betas, int ndof,
                                      const int* dof_kind, const int* dof_body, const double* dof_dir,
                                      const double* dof_axis, int nforce, const int* force_kind, const int* force_body,
                                      const double* force_dir, const double* force_axis, double* nvel_device,
                                      double* nds_device, double* fk_device, void* stream);

/* Resident bodies and cross-body batches. The reference solves one body per
 * run, its problems one after another (Solver/NEMOH.f90:129-143, the boundary
 * SOLVE_POTENTIAL_*_DIRECT once per problem); these entry points extend that
 * boundary to many bodies at once:
 *
 * nemoh_b200_add_body keeps a body on the device for the life of the context:
 * its mesh (as nemoh_b200_set_mesh, INITIALIZE + PRE_PROC_MESH), environment
 * and generalised normals nds (nint x 2^s nfa, Integration.dat), and its own
 * NQ state. body_id receives its index (0, 1, ...). The context's current mesh
 * (set_mesh) is not changed.
 *
 * nemoh_b200_solve_bodies solves nitem (body[i], omegas[i]) items, each with
 * nrhs (1..16) right-hand sides, as nemoh_b200_solve_frequencies does for one
 * body: nvel holds, item after item, (2^s nfa_i) x nrhs complex NVEL columns;
 * force receives, item after item, nint_i x nrhs complex forces. Items of
 * different bodies share one launch sequence (systems of different orders in
 * one batch); the items of one body are set up in the order given (its NQ
 * state follows them). Batches are sized by free device memory. */
int nemoh_b200_add_body(nemoh_ctx* ctx, int np, int nfa, int nsymy, const double* xyz, const int* m1234, double rho,
                        double g, double depth, int nint, const double* nds, int* body_id);
int nemoh_b200_body_count(const nemoh_ctx* ctx);
int nemoh_b200_solve_bodies(nemoh_ctx* ctx, int nitem, const int* body, const double* omegas, int nrhs,
                            const double* nvel, double* force);
/* CUDA graphs for repeated cross-body batches (on = 1; off by default). In
 * graph mode every batch of nemoh_b200_solve_bodies / _solve_requests does
 * its host setup and uploads first and then issues its launch sequence, which
 * reads device buffers only; the second batch with the same sequence (same
 * bodies' orders and depth regimes in the same order, nrhs, buffers and
 * pointers) is captured into a graph and later ones replay it. Refinement
 * passes beyond the REFINE_CHUNK captured ones and the FP64 fallback run as
 * ordinary launches after the replay. The timings of nemoh_b200_last_timings
 * then hold the whole batch in solve_ms (assembly and factor 0).
 * nemoh_b200_graph_stats: graphs captured and replayed so far. */
int nemoh_b200_set_graphs(nemoh_ctx* ctx, int on);
int nemoh_b200_graph_stats(const nemoh_ctx* ctx, long long* captures, long long* replays);

/* Evaluates now, for every resident body, the frequency-independent Rankine
 * part of each depth regime it can meet (deep water; finite depth when its
 * depth is finite), which a solve otherwise evaluates at the body's first
 * frequency of that regime (kept within the resident bodies' cache budget).
 * A server calls it once after adding its bodies, so that no request pays
 * for it. */
int nemoh_b200_prepare_bodies(nemoh_ctx* ctx);
/* Autotuning of the triangular sweep (process-wide; on by default). Off, a
 * batch shape not tuned yet is solved with the default sweep instead of
 * timing the candidates first. */
int nemoh_b200_set_autotune(int on);

/* Serving requests on resident bodies. nemoh_b200_set_body_dofs gives a body
 * its ndof radiation DOFs (kind, dir, axis as in nemoh_b200_body_conditions;
 * 1 + ndof <= 16). nemoh_b200_solve_requests solves nreq (body[i], omegas[i],
 * betas[i] in radians) requests with right-hand sides built on the device by
 * the pre-processor's formulas (preProcessor/BodyConditions.f90:27-137,
 * Environment.f90:86-100; wave measurement point at the origin): per request
 * the diffraction problem at its heading, then the radiation DOFs; force
 * receives, request after request, nint_i x (1 + ndof) complex forces. The
 * bodies of one call must have the same ndof. */
int nemoh_b200_set_body_dofs(nemoh_ctx* ctx, int body, int ndof, const int* dof_kind, const double* dof_dir,
                             const double* dof_axis);
int nemoh_b200_solve_requests(nemoh_ctx* ctx, int nreq, const int* body, const double* omegas, const double* betas,
                              double* force);
/* Same with nvel and force in device memory of the context's device, ordered
 * on `stream` (cudaStream_t) like nemoh_b200_solve_frequencies_device. */
int nemoh_b200_solve_bodies_device(nemoh_ctx* ctx, int nitem, const int* body, const double* omegas, int nrhs,
                                   const double* nvel_device, double* force_device, void* stream);

/* No counterpart in the reference: an entry point that allocates nothing, for
 * hosts whose device memory is held by their own allocator (a PyTorch caching
 * allocator, a batching server that admits work by free HBM) and for hosts
 * whose other streams must not be stalled by cudaFree's device-wide sync.
 * Factors in place (FP64 LU without pivoting, as the context path) and solves
 * nsys dense complex systems resident on `device`:
 *   a_device: nsys x (n x n) complex, column-major, overwritten by L\U;
 *   x_device: nsys x nrhs x n complex, right-hand sides in, solutions out;
 *   1 <= nrhs <= 16; both pointers 16-byte aligned; stream = cudaStream_t.
 * Scratch comes from one static device array of NEMOH_B200_NOALLOC_SCRATCH_BYTES
 * (16 MiB) per device: a call needing more (about
 * nsys*(48 KiB + ceil(n/64)*128 KiB + 16*n*nrhs) bytes) returns
 * NEMOH_B200_ECAPACITY. The first call on a device does a one-time set-up
 * (symbol lookup, kernel attributes) and should come before any stream
 * capture. All calls on a device share the scratch, so calls that overlap on
 * the GPU race. Both pointers must be device (or managed) memory of `device`:
 * host memory or another GPU's memory is refused with NEMOH_B200_EINVAL before
 * any launch. The scratch address found at set-up is kept for the life of the
 * process; after cudaDeviceReset on that device it is stale, so do not call
 * this entry point again in a process that reset the device. The call returns
 * after its work on `stream` has finished; msg (may be NULL) receives the
 * error text. */
#define NEMOH_B200_NOALLOC_SCRATCH_BYTES (16u << 20)
int nemoh_b200_factor_solve_device_noalloc(int device, int n, int nsys, double* a_device, int nrhs, double* x_device,
                                           void* stream, char* msg, int msg_len);

/* Diagnostics used by the parity tests. */
/* influence matrices of one frequency (each nfa x nfa complex, column-major):
 * dp/dm = ZIJ of symmetry class +/-, sp/sm = single-layer S+/S- (SP1+i SP2, SM1+i SM2);
 * depth_mode = 1 if the finite-depth Green function was used. */
int nemoh_b200_assemble(nemoh_ctx* ctx, double omega, double* dp, double* dm, double* sp, double* sm,
                        int* depth_mode);
/* xr[328], xz[46], apd[4*328*46] = APD1X, APD1Z, APD2X, APD2Z column-major (I,J) */
int nemoh_b200_get_tables(nemoh_ctx* ctx, double* xr, double* xz, double* apd);
/* out[8*nfa] = XN,YN,ZN,XG,YG,ZG,AIRE,TDIS; zer = ZER */
int nemoh_b200_get_geometry(nemoh_ctx* ctx, double* out, double* zer);
/* timing of the last solve_frequencies call: assembly, factorization, solve+potential+forces (ms) */
int nemoh_b200_last_timings(nemoh_ctx* ctx, double* assemble_ms, double* factor_ms, double* solve_ms);
/* the factorization alone within factor_ms (the rest of factor_ms is the
 * triangular solves, and in mixed precision the refinement) */
int nemoh_b200_last_factor_ms(nemoh_ctx* ctx, double* lu_ms);
/* mixed precision: refinement iterations and final max relative residual of the
 * last solve; iterations = -1 when the refinement did not reach 1e-12 (FP32
 * factors too inaccurate, e.g. near an irregular frequency) and that batch was
 * factored and solved again in FP64 on the device */
int nemoh_b200_last_refinement(nemoh_ctx* ctx, int* iterations, double* residual);
/* mixed precision: batches that needed the FP64 fallback since the context was
 * created, and the systems re-solved there (a batch of several bodies
 * re-solves only its systems that missed the tolerance; systems counts only
 * those partial fallbacks) */
int nemoh_b200_fallback_count(const nemoh_ctx* ctx, long long* batches, long long* systems);
/* number of CUDA kernel launches issued by this context since creation */
long long nemoh_b200_launch_count(const nemoh_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* NEMOH_B200_H */
