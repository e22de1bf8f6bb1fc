/*
 * meanas_fdfd.h -- C ABI of the B200 FDFD solve path (libmeanas_fdfd.so).
 *
 * Drop-in for the hot path behind meanas.fdfd.solvers.generic()
 * (reference: meanas/fdfd/solvers.py:66-141): the E-field wave operator
 *     A0 = pe (ch pm mu^-1 ce - omega^2 eps) pe          (meanas/fdfd/operators.py:40-96)
 * applied matrix-free on the Yee grid, its symmetrised form Pl A0 Pr
 * (meanas/fdfd/operators.py:99-123), and the Krylov solve of A0 E = -i omega J.
 *
 * Conventions
 *   - Fields are 3 x X x Y x Z, C order (z fastest), as meanas.fdmath.vec() makes
 *     them (meanas/fdmath/vectorization.py:51-68); N = X*Y*Z cells, 3N elements.
 *   - Complex arrays are interleaved (re, im): complex128 = 2 doubles,
 *     complex64 = 2 floats.
 *   - Every pointer to a field or table is DEVICE memory of the current CUDA
 *     device; `stream` is a cudaStream_t (NULL = legacy default stream).
 *   - No function allocates device memory: callers size and pass workspaces.
 *   - Return codes: 0 = success; > 0 = the solver stopped without meeting its
 *     tolerance (an FDFD_STATUS_* value); < 0 = argument or CUDA error, with the
 *     message available from fdfd_last_error() (per calling thread).
 */
#ifndef MEANAS_FDFD_H
#define MEANAS_FDFD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDFD_ABI_VERSION 1

/* solver status (fdfd_solve_info.status and positive return codes) */
#define FDFD_STATUS_CONVERGED 1
#define FDFD_STATUS_MAXITER 2
#define FDFD_STATUS_BREAKDOWN 3
#define FDFD_STATUS_NONFINITE 4

/* error codes (negative returns) */
#define FDFD_ERR_ARG (-1)
#define FDFD_ERR_CUDA (-2)
#define FDFD_ERR_WORKSPACE (-3)

/* fdfd_grid_desc.flags */
#define FDFD_GRID_FP32 1 /* also build complex64 tables (needed by FDFD_METHOD_MIXED) */

/* operators for fdfd_apply */
#define FDFD_OP_A0 0      /* y = A0 x                                        */
#define FDFD_OP_SYM 1     /* y = Pl A0 Pr x  (the matrix generic() hands QMR) */
#define FDFD_OP_SYM_H 2   /* y = (Pl A0 Pr)^H x  (generic(adjoint=True))     */

/* precisions */
#define FDFD_C128 0
#define FDFD_C64 1

/* solver methods */
#define FDFD_METHOD_COCG 0     /* complex128 COCG on the symmetrised system            */
#define FDFD_METHOD_MIXED 1    /* complex64 BiCGSTAB inner + complex128 refinement     */
#define FDFD_METHOD_BICGSTAB 2 /* complex128 BiCGSTAB                                  */

/* stopping criteria */
#define FDFD_CRIT_TRUE 0    /* ||b0 - A0 E|| <= max(rtol ||b0||, atol), b0 = -i omega J      */
#define FDFD_CRIT_PRECOND 1 /* scipy's test on the symmetrised system generic() builds:
                               ||Pl (b0 - A0 E)|| <= max(rtol ||Pl b0||, atol)            */

typedef struct fdfd_plan fdfd_plan;

/* Grid, material and frequency: the arguments of generic() that define A0. */
typedef struct fdfd_grid_desc {
  int32_t shape[3];     /* X, Y, Z (each >= 1)                                     */
  int32_t flags;        /* FDFD_GRID_*                                             */
  double omega[2];      /* complex angular frequency (re, im)                      */
  const void* dxe[3];   /* complex128[shape[a]]: dxes[0][a] (E-grid cell widths)   */
  const void* dxh[3];   /* complex128[shape[a]]: dxes[1][a] (H-grid cell widths)   */
  const void* inv_dxe[3]; /* optional complex128 1/dxe (NULL: computed on device)  */
  const void* inv_dxh[3]; /* optional complex128 1/dxh                             */
  const double* epsilon;  /* float64[3N]; referenced, not copied: keep it alive    */
  const double* mu;       /* float64[3N] or NULL (mu = 1)                          */
  const double* pec;      /* float64[3N] or NULL; nonzero = PEC on that E component */
  const double* pmc;      /* float64[3N] or NULL; nonzero = PMC on that H component */
} fdfd_grid_desc;

typedef struct fdfd_solve_opts {
  int32_t method;        /* FDFD_METHOD_*                                           */
  int32_t criterion;     /* FDFD_CRIT_*                                             */
  int32_t adjoint;       /* nonzero: solve A0^H E = -i omega J (generic(adjoint=True)) */
  int32_t maxiter;       /* Krylov iteration cap (inner iterations summed for MIXED) */
  double rtol;
  double atol;
  int32_t has_guess;     /* nonzero: E holds an initial guess on entry (E_guess)    */
  int32_t chunk;         /* iterations per launch batch / CUDA graph (0 = default)  */
  int32_t use_graph;     /* nonzero: replay iteration batches as CUDA graphs        */
  int32_t max_outer;     /* MIXED: refinement steps cap (0 = default)               */
  double inner_rtol;     /* MIXED: residual reduction per inner solve (0 = default) */
  double* history;       /* optional device float64[maxiter + 1]: relative residuals */
  int32_t profile;       /* nonzero: time every iteration kernel with CUDA events (no
                            graphs); fills the *_ms / *_launches fields of the info  */
  int32_t pad_;
} fdfd_solve_opts;

typedef struct fdfd_solve_info {
  int32_t status;          /* FDFD_STATUS_*                                          */
  int32_t iterations;      /* Krylov iterations (inner iterations summed for MIXED)  */
  int32_t outer_iterations;/* MIXED refinement steps                                 */
  int32_t kernel_launches; /* kernels launched by this call                          */
  double residual;         /* ||b0 - A0 E|| / ||b0||, FP64, recomputed at the end    */
  double residual_pc;      /* ||Pl (b0 - A0 E)|| / ||Pl b0||                         */
  /* with opts->profile: device time of the iteration kernels, by kind
     [0] COCG stencil pass  [1] COCG pointwise pass
     [2] BiCGSTAB P pass    [3] BiCGSTAB S pass        (ms summed, launch counts) */
  double kernel_ms[4];
  int32_t kernel_count[4];
} fdfd_solve_info;

/* Version of this ABI (FDFD_ABI_VERSION). */
int fdfd_abi_version(void);

/* Message of the last error on the calling thread ("" if none). */
const char* fdfd_last_error(void);

/* Device bytes the plan keeps (1/mu, packed PEC/PMC bits, 1D tables, complex64
 * copies when FDFD_GRID_FP32 is set).  Replaces the sparse assembly of
 * meanas/fdfd/operators.py:76-96 (no matrix is ever stored). */
int fdfd_plan_workspace_bytes(const fdfd_grid_desc* desc, size_t* bytes);

/* Build a plan in caller-provided device memory `ws` (>= fdfd_plan_workspace_bytes,
 * 256-byte aligned).  Enqueues its set-up kernels on `stream`. */
int fdfd_plan_create(const fdfd_grid_desc* desc, void* ws, size_t ws_bytes, void* stream,
                     fdfd_plan** out);

/* Refill an existing plan from a new description of the same shape, flags and set of
 * optional arrays (new omega, cell widths, epsilon, mu, masks), on `stream`.  The
 * plan keeps its workspace and tiling, so iteration graphs captured for it stay valid
 * when the array pointers are unchanged.  Used by the serving loop, whose slots
 * serve request after request of one grid size (no counterpart in the reference). */
int fdfd_plan_update(fdfd_plan* plan, const fdfd_grid_desc* desc, void* stream);

/* Release the host-side plan object (the caller owns `ws`). */
int fdfd_plan_destroy(fdfd_plan* plan);

/* Override the x-planes-per-CTA tiling for one precision (autotuner hook). */
int fdfd_plan_set_xchunk(fdfd_plan* plan, int32_t precision, int32_t xchunk);

/* Matrix-free operator product y = op(x) in complex128 or complex64 (x, y: 3N).
 * FDFD_OP_A0 replaces operators.e_full(...) @ x (meanas/fdfd/operators.py:40-96);
 * FDFD_OP_SYM replaces (Pl @ A0 @ Pr) @ x (meanas/fdfd/solvers.py:116-125);
 * FDFD_OP_SYM_H replaces (Pl @ A0 @ Pr).H @ x (meanas/fdfd/solvers.py:119-122). */
int fdfd_apply(fdfd_plan* plan, int32_t op, int32_t precision, const void* x, void* y, void* stream);

/* Device workspace bytes fdfd_solve needs for these options. */
int fdfd_solve_workspace_bytes(const fdfd_plan* plan, const fdfd_solve_opts* opts, size_t* bytes);

/* Solve A0 E = -i omega J (or the adjoint) for E (complex128, 3N).
 * Replaces meanas/fdfd/solvers.py:66-141 (generic) with its default
 * matrix_solver _scipy_qmr (:21-63).  J: complex128[3N].  E: complex128[3N]
 * output (and initial guess when opts->has_guess).  Synchronous with respect to
 * the host (it polls the device for convergence); all work runs on `stream`. */
int fdfd_solve(fdfd_plan* plan, const fdfd_solve_opts* opts, const void* J, void* E, void* ws,
               size_t ws_bytes, fdfd_solve_info* info, void* stream);

/* FP64 residual norms of a field: out[0] = ||b0 - A0 E||, out[1] = ||Pl (b0 - A0 E)||,
 * out[2] = ||b0||, out[3] = ||Pl b0|| with b0 = -i omega J
 * (the check of meanas/test/test_fdfd.py:14-18).  `ws` >= fdfd_residual_workspace_bytes.
 * The results pass through the plan's pinned host state, so calls on one plan
 * (fdfd_residual, fdfd_residual_static, fdfd_solve) must not run at the same time from
 * different host threads. */
int fdfd_residual_workspace_bytes(const fdfd_plan* plan, size_t* bytes);
int fdfd_residual(fdfd_plan* plan, const void* E, const void* J, double out[4], void* ws,
                  size_t ws_bytes, void* stream);

/* dL/d(epsilon) from the forward field E and the adjoint field E_adj
 * (fdfd_solve with adjoint = 1 and J_adj = dL/dE* / (-i omega), torch's convention
 * grad = 2 dL/dE*): grad[i] = Re(omega^2 conj(E_adj[i]) E[i]), zero on PEC components.
 * No counterpart function in the reference, which assembles this from generic() and
 * generic(adjoint=True) (meanas/fdfd/solvers.py:119-137); grad: float64[3N]. */
int fdfd_eps_gradient(fdfd_plan* plan, const void* E, const void* E_adj, double* grad, void* stream);

/* fdfd_e2h flags */
#define FDFD_E2H_CONJ 1 /* S = E x conj(H) instead of E x H */
#define FDFD_E2H_H_IN 2 /* H is an input: only S is computed, from E and the caller's H */

/* The step after the solve: H = e2h(omega, dxes, mu, pmc) @ E
 * (meanas/fdfd/operators.py:253-282: pm diag(1/mu) ce(E) / (-i omega)) into H, and when
 * S is not NULL the Yee-grid cross product S = E x H (functional.poynting_e_cross_h,
 * meanas/fdfd/functional.py:187-221) or, with FDFD_E2H_CONJ, S = E x conj(H) (the
 * poynting_e_cross(E) @ H.conj() of meanas/fdfd/operators.py:310-336 that
 * meanas/test/test_fdfd.py:38-40 forms; Re(S)/2 is the time-averaged Poynting vector).
 * With FDFD_E2H_H_IN, H is read instead of computed.  E, H, S: complex128 [3N] device
 * arrays; H may be NULL when only S is wanted. */
int fdfd_e2h(fdfd_plan* plan, const void* E, void* H, void* S, int32_t flags, void* stream);

/* fdfd_tfsf_source flags */
#define FDFD_SRC_EDGES 1    /* e_boundary_source: keep J only where shifting Q changes it */
#define FDFD_SRC_PERIODIC 2 /* with FDFD_SRC_EDGES: periodic_mask_edges = True */

/* The step before the solve: J = e_tfsf_source(Q, omega, dxes, epsilon, mu) @ E
 * (meanas/fdfd/operators.py:366-393: (A0 Q - Q A0) E / (-i omega), A0 = e_full without
 * masks, Q = diag(tf_region)), or with FDFD_SRC_EDGES
 * e_boundary_source(Q, ..., periodic_mask_edges) @ E (:396-450).  The plan must have no
 * PEC/PMC (the reference's source operators take none).  E, J: complex128 [3N] device
 * arrays (J must not alias E); tf_region: float64 [3N]. */
int fdfd_tfsf_source(fdfd_plan* plan, const void* E, const double* tf_region, void* J, int32_t flags,
                     void* stream);

/* A waveguide cross-section and the half-space of a unidirectional mode source
 * (the `axis`, `polarity` and `slices` arguments of meanas/fdfd/waveguide_3d.py). */
typedef struct fdfd_mode_slice {
  int32_t axis;           /* propagation axis, 0..2                                       */
  int32_t polarity;       /* +1 or -1                                                     */
  int32_t lo[3], hi[3];   /* slices as [lo, hi) per axis; hi[axis] = lo[axis] + 1          */
  int32_t mask_lo, mask_hi; /* planes of the source's half-space mask along the axis       */
} fdfd_mode_slice;

/* expand_e (meanas/fdfd/waveguide_3d.py:206-257): E_out[c, .., i, ..] = phase[i] *
 * E_mode[c, .., lo[axis], ..] inside the transverse window, 0 outside; phase =
 * exp(-i polarity wavenumber r_E) per plane of the axis (complex128[n_axis]).  With
 * mask_out (float64 [3N], may be NULL) also the half-space mask of compute_source
 * (1 on planes [mask_lo, mask_hi)).  E_mode, E_out: complex128 [3N] device arrays. */
int fdfd_mode_expand(fdfd_plan* plan, const void* E_mode, const void* phase, const fdfd_mode_slice* slice,
                     void* E_out, double* mask_out, void* stream);

/* The unidirectional mode source J = waveguide_3d.compute_source(E_mode, wavenumber,
 * omega, dxes, axis, polarity, slices, epsilon, mu) (meanas/fdfd/waveguide_3d.py:113-156):
 * fdfd_mode_expand into E_work / mask_work, then e_boundary_source(mask) @ E_work
 * (fdfd_tfsf_source with FDFD_SRC_EDGES).  The plan holds omega, dxes, epsilon, mu and
 * no PEC/PMC.  E_work (complex128 [3N]) and mask_work (float64 [3N]) are caller scratch;
 * J: complex128 [3N]. */
int fdfd_mode_source(fdfd_plan* plan, const void* E_mode, const void* phase, const fdfd_mode_slice* slice,
                     void* E_work, double* mask_work, void* J, void* stream);

/* A general complex128 CSR matrix (device arrays), as scipy.sparse.csr_array holds it:
 * row r's nonzeros are data[indptr[r] .. indptr[r+1]) at columns indices[...]. */
typedef struct fdfd_csr_desc {
  int64_t n;              /* rows = columns (< 2^31)                    */
  int64_t nnz;
  const int64_t* indptr;  /* int64[n + 1]                               */
  const int32_t* indices; /* int32[nnz]                                 */
  const void* data;       /* complex128[nnz]                            */
} fdfd_csr_desc;

/* y = A x for a CSR matrix (x, y: complex128[n], distinct). */
int fdfd_csr_spmv(const fdfd_csr_desc* A, const void* x, void* y, void* stream);

/* Workspace bytes of fdfd_csr_solve (7 complex128[n] vectors + scalar state). */
int fdfd_csr_solve_workspace_bytes(const fdfd_csr_desc* A, size_t* bytes);

/* Solve A x = b for a general CSR matrix with complex128 BiCGSTAB: the reference's
 * second plugin point, matrix_solver(A, b, **opts) -> x (meanas/fdfd/solvers.py:97-103,134,
 * whose default _scipy_qmr is :21-63).  Stops when ||r|| <= max(rtol ||b||, atol) on the
 * recurrence residual (scipy's rule) or after opts->maxiter iterations; uses rtol, atol,
 * maxiter and has_guess (x holds x0 on entry) of `opts`.  info->residual is the true
 * ||b - A x|| / ||b|| of the returned x, which is the last iterate whatever the status. */
int fdfd_csr_solve(const fdfd_csr_desc* A, const fdfd_solve_opts* opts, const void* b, void* x, void* ws,
                   size_t ws_bytes, fdfd_solve_info* info, void* stream);

/* ---- FDTD (time domain) ----
 * The Yee updates of meanas/fdtd: maxwell_h / maxwell_e (meanas/fdtd/base.py:13-125) and
 * updates_with_cpml (meanas/fdtd/pml.py:115-230), on real fields of 3 x X x Y x Z
 * (float32 or float64), with the arithmetic of the reference step by step, so results are
 * the same bits. */
#define FDFD_REAL64 0
#define FDFD_REAL32 1
#define FDFD_FDTD_PLAIN 0 /* maxwell_h / maxwell_e                   */
#define FDFD_FDTD_CPML 1  /* updates_with_cpml (CPML on the faces set) */

typedef struct fdfd_fdtd_face {
  int32_t thickness;      /* PML layers on this face, 0 = none                            */
  int32_t pad_;
  const double* param_e;  /* float64[3][thickness]: p0, p1, p2 of the E update (cpml_params) */
  const double* param_h;  /* the same for the H update                                    */
  void* psi_e[2];         /* psi of the E update, two transverse components, psi_type,     */
  void* psi_h[2];         /* each of the face region's shape (thickness along the axis)    */
} fdfd_fdtd_face;

typedef struct fdfd_fdtd_desc {
  int32_t shape[3];
  int32_t field_type;     /* FDFD_REAL64 / FDFD_REAL32                                    */
  int32_t psi_type;       /* FDFD_REAL64 / FDFD_REAL32 (updates_with_cpml's dtype)         */
  int32_t form;           /* FDFD_FDTD_PLAIN / FDFD_FDTD_CPML                              */
  double dt;
  const double* dxe[3];   /* float64[shape[a]]: dxes[0][a]                                 */
  const double* dxh[3];   /* float64[shape[a]]: dxes[1][a]                                 */
  const double* epsilon;  /* float64[3N]                                                   */
  const double* mu;       /* float64[3N] or NULL (mu = 1)                                  */
  fdfd_fdtd_face face[3][2]; /* [axis][0: low face (polarity -1), 1: high face (+1)]      */
} fdfd_fdtd_desc;

/* H half step: maxwell_h(dt, dxes)(E, H, mu) or updates_with_cpml's update_H(E, H, mu). */
int fdfd_fdtd_update_h(const fdfd_fdtd_desc* desc, const void* E, void* H, void* stream);
/* E half step: maxwell_e(dt, dxes)(E, H, epsilon) or update_E(E, H, epsilon). */
int fdfd_fdtd_update_e(const fdfd_fdtd_desc* desc, void* E, const void* H, void* stream);

/* fdfd_residual without a workspace, for callers that cannot allocate device memory
 * (an exhausted or frozen allocator, or a host program that owns every device buffer
 * and can pass only inputs and outputs).  No counterpart in the reference.
 * The reduction scratch is a fixed 1 MiB array inside the library, held by every
 * device that loads it until exit; grids needing more than 32752 partial sums (one per
 * 8-plane block of a 32 x 8 y/z tile, about 2048 cells each) are rejected with
 * FDFD_ERR_ARG.  The first call on a device looks up that array's device
 * address; make it before any stream capture.  All calls share the array: calls
 * whose work overlaps on the GPU (other streams, other threads) race on it.
 * Like fdfd_residual, the four results pass through the plan's pinned host state:
 * calls on one plan (this one, fdfd_residual, fdfd_solve) must not run at the same
 * time from different host threads, even on one stream.  The looked-up address is
 * kept for the life of the process: the library must not be used on a device after
 * that device has been reset (cudaDeviceReset) in the same process.
 * Allocates nothing; same results as fdfd_residual. */
int fdfd_residual_static(fdfd_plan* plan, const void* E, const void* J, double out[4], void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MEANAS_FDFD_H */
