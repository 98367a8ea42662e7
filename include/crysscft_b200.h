/*
 * crysscft_b200.h — C ABI of the B200 pseudo-spectral propagator library.
 *
 * The library replaces the reference's diffusion-solver plugin
 * (class CrysPSSolverBase, src/solver_base.h:8-51, and its three
 * implementations CrysPSSolverP1, CrysPSSolver3m, CrysPSSolverPmmm) and the
 * contour/iteration loop that drives it (src/crysSCFT_sample.cpp:373-531).
 * Every entry point takes plain pointers and sizes and returns an int status
 * (SCFT_OK == 0).  Host pointers are ordinary (pageable or pinned) memory;
 * "_device" entry points take device pointers on the solver's GPU and an
 * optional cudaStream_t passed as void* (NULL = the solver's own stream).
 *
 * Grids are C-ordered (x slowest, z fastest) like the reference.  "Logical"
 * sizes are the full-cell grid (Nx, Ny, Nz); "physical" sizes are what the
 * solver stores: the full grid for P1, (Nx/2, Ny/2, Nz/2) for 3M and PMMM.
 *
 * Thread safety: one handle must not be used from two host threads at once
 * (the reference's solvers are not thread-safe either).
 */
#ifndef CRYSSCFT_B200_H
#define CRYSSCFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference prints "ERROR" and calls exit(1)) ---- */
#define SCFT_OK 0
#define SCFT_ERR_INVALID_ARG 1   /* null handle/pointer, bad kind, bad direction */
#define SCFT_ERR_BAD_GRID 2      /* grid rejected (src/solver_p1.h:101-108, solver_3m.h:81-92, solver_Pmmm.h:71-82) */
#define SCFT_ERR_CUDA 3          /* a CUDA runtime call failed; see scft_last_error() */
#define SCFT_ERR_ALLOC 4         /* device or pinned allocation failed */
#define SCFT_ERR_NOT_READY 5     /* set_cell_para / set_contour_step / fields not set yet */
#define SCFT_ERR_NUMERIC 6       /* NaN/Inf or Q <= 0 detected in an iteration */
#define SCFT_ERR_TIMEOUT 7       /* a bounded device-side wait gave up */
#define SCFT_ERR_UNSUPPORTED 8   /* valid request this build does not implement */
#define SCFT_ERR_NO_DEVICE 9     /* no CUDA device / extension unusable */

/* ---- solver kinds: the reference's three CrysPSSolverBase classes ---- */
#define SCFT_SOLVER_P1 0   /* CrysPSSolverP1     src/solver_p1.h:14-214  */
#define SCFT_SOLVER_3M 1   /* CrysPSSolver3m     src/solver_3m.h:14-324  */
#define SCFT_SOLVER_PMMM 2 /* CrysPSSolverPmmm   src/solver_Pmmm.h:13-215 */

/* ---- arithmetic of the triplets ---- */
#define SCFT_FP64 0 /* plain form: FP64 everywhere (the reference's arithmetic) */
#define SCFT_FP32 1 /* FP32 triplets; Q, phi, energy and mixing stay FP64 */

typedef struct scft_solver_s* scft_solver_t;
typedef struct scft_diblock_s* scft_diblock_t;
typedef struct scft_batch_s* scft_batch_t;

/* Text of the last error on this host thread (static storage, never NULL). */
const char* scft_last_error(void);
/* Short name of a status code. */
const char* scft_status_string(int status);
/* Library version string. */
const char* scft_version(void);

/* ========================================================================
 * Solver plugin: replaces CrysPSSolverBase and its implementations.
 * ======================================================================== */

/* Constructor.  Replaces CrysPSSolverP1(grid) (src/solver_p1.h:16-19),
 * CrysPSSolver3m(grid, translational_part) (src/solver_3m.h:17-20) and
 * CrysPSSolverPmmm(grid) (src/solver_Pmmm.h:16-19).  translational_part
 * (9 doubles, may be NULL = zeros) is used by SCFT_SOLVER_3M only: the
 * translations, in cell fractions, of the mirrors normal to z (g[0..2]), y (g[3..5])
 * and x (g[6..8]), as in generate_m3_operation (src/solver_utilities.h:56-66).
 * Accepted are the translations for which each mirror maps the even sub-lattice onto
 * another parity class of the grid: components along other axes 0 or 1/2 (1/2 needs
 * N % 4 == 0 on that axis), the component along the mirror normal an even number of
 * grid points; anything else returns SCFT_ERR_INVALID_ARG.  Half-cell components make
 * the triplet a sum of Kronecker products (see scft_operator_terms), which runs on the
 * per-axis kernels instead of the persistent contour kernel.
 * device: CUDA ordinal (-1 = current device). */
int scft_solver_create(int kind, const size_t grid_size_log[3], const double translational_part[9],
                       int precision, int device, scft_solver_t* out);
/* Destructor (~CrysPSSolverP1 etc.).  NULL is accepted.  While iteration contexts
 * (scft_diblock_t) built on the solver exist, the solver stays alive and is freed with
 * the last of them, so the two may be destroyed in either order. */
int scft_solver_destroy(scft_solver_t solver);

/* Host-only, no device work (callable on a machine without a GPU): the per-axis
 * factors of the triplet the solver of `kind` builds for grid_size_log,
 * translational_part (as in scft_solver_create), cell lengths cell[0..2] (used as
 * given, also for PMMM) and contour step ds.  The triplet on the physical grid is
 * sum_t A_x^t (x) A_y^t (x) A_z^t.  *nterms receives the number of terms; when
 * `factors` is not NULL it receives, term after term, A_x^t, A_y^t, A_z^t (row-major,
 * n_a x n_a with n_a the physical axis length), provided `capacity` (doubles) holds
 * them all.  No counterpart in the reference, which never forms these matrices
 * (its triplets are src/solver_p1.h:184-202, src/solver_3m.h:281-324,
 * src/solver_Pmmm.h:194-215). */
int scft_operator_terms(int kind, const size_t grid_size_log[3], const double translational_part[9],
                        const double cell[3], double ds, size_t* nterms, double* factors, size_t capacity);

/* CrysPSSolverBase::set_cell_para (src/solver_base.h:16): {Lx,Ly,Lz,alpha,beta,gamma}.
 * As in the reference, PMMM uses cell_para[0] for all three axes
 * (src/solver_Pmmm.h:98-104); P1 and 3M use cell_para[0..2]. */
int scft_solver_set_cell_para(scft_solver_t solver, const double cell_para[6]);
/* PMMM with an orthorhombic cell: after enable = 1, set_cell_para uses Lx, Ly, Lz
 * (cell_para[0..2]) instead of the reference's cubic cell_para[0] (src/solver_Pmmm.h:101).
 * No counterpart in the reference; validated against P1 and 3M on the same cell. */
int scft_solver_set_pmmm_anisotropic(scft_solver_t solver, int enable);
/* CrysPSSolverBase::set_contour_step (src/solver_base.h:18).  Operators are cached per ds. */
int scft_solver_set_contour_step(scft_solver_t solver, double ds);

/* Getters of src/solver_base.h:22-27. */
int scft_solver_get_grid_size_log(scft_solver_t solver, size_t out[3]);
int scft_solver_get_grid_size_phy(scft_solver_t solver, size_t out[3]);
int scft_solver_get_space_size_phy(scft_solver_t solver, size_t* out);
int scft_solver_get_cell_para(scft_solver_t solver, double out[6]);
int scft_solver_get_ds(scft_solver_t solver, double* out);

/* CrysPSSolverBase::get_iomat_for_diffusion (src/solver_base.h:28): a host buffer of
 * space_size_phy doubles owned by the solver (pinned), which diffusion() transforms in place. */
int scft_solver_get_iomat_for_diffusion(scft_solver_t solver, double** out);
/* CrysPSSolverBase::diffusion (src/solver_base.h:20): one triplet on the host iomat
 * (copy to the GPU, triplet, copy back; synchronous). */
int scft_solver_diffusion(scft_solver_t solver);
/* One triplet in place on a device buffer of space_size_phy elements (FP64). */
int scft_solver_diffusion_device(scft_solver_t solver, double* d_io, void* stream);

/* solve_diffusion_equation (src/crysSCFT_sample.cpp:373-396) on device buffers:
 * q has (Ns+1)*space_size_phy doubles; direction +1 fills slots 0..Ns, -1 fills Ns..0;
 * every step is q <- wds * T(wds * q). */
int scft_solver_propagate_device(scft_solver_t solver, double* d_q, const double* d_init,
                                 const double* d_wds, size_t Ns, int direction, void* stream);
/* The same on host buffers (copies in and out; synchronous). */
int scft_solver_propagate(scft_solver_t solver, double* q, const double* init, const double* wds,
                          size_t Ns, int direction);

/* ========================================================================
 * AB-diblock SCFT iteration: replaces diblock_scft_simple_iterate
 * (src/crysSCFT_sample.cpp:426-531) and its helpers (:294-424).
 * ======================================================================== */

/* Parameters as in the reference driver: NsA = size_t(fA/ds), NsB = size_t((1-fA)/ds)
 * (src/crysSCFT_sample.cpp:442-444); both must be >= 1.  The solver must have its cell
 * set; create() calls set_contour_step(ds). */
int scft_diblock_create(scft_solver_t solver, double fA, double ds, double xN, double acceptance,
                        scft_diblock_t* out);
int scft_diblock_destroy(scft_diblock_t d);
int scft_diblock_get_contour_counts(scft_diblock_t d, size_t* NsA, size_t* NsB);
/* The solver the context was created on (the handle stays owned by its creator, or by the
 * batch for scft_batch_instance contexts); its getters give the grid and space size. */
int scft_diblock_get_solver(scft_diblock_t d, scft_solver_t* out);

/* Load wA, wB (space_size_phy doubles each, host). */
int scft_diblock_set_fields(scft_diblock_t d, const double* wA, const double* wB);
/* Copy phiA, phiB (of the last iteration) and wA, wB (after its update) to host; any may be NULL. */
int scft_diblock_get_fields(scft_diblock_t d, double* phiA, double* phiB, double* wA, double* wB);
/* Backward pass of the differentiation form, from the stored contour of the last
 * iteration (FP64, or the FP32 contour of a precision-form iteration: its slices and
 * Boltzmann factors are promoted, the derivative triplets and sums run in FP64, so the
 * result is the precision form's own stress): dlnQ_dL[a] = d ln Q / d L_a at fixed fields, by the adjoint identity
 * dQ/dL_a = (1/M) sum_t < q+[t+1], D_t (dT/dL_a) D_t q[t] > (one term per contour step;
 * T = A_x (x) A_y (x) A_z, so dT/dL_x = (dA_x/dL_x) (x) A_y (x) A_z).  The stress
 * dF/dL_a equals -dlnQ_dL[a] at the SCFT saddle point (there dF/dphi = 0).  For PMMM
 * (cubic cell in the reference) the three axis derivatives are still reported; the
 * cubic dF/dL is minus their sum.  dF_dxN = dF/dchiN at fixed fields, from the energy
 * terms of print_energy (src/crysSCFT_sample.cpp:404-418): <phiA phiB> +
 * <1 - phiA - phiB>/2.  Q_out: the Q of that iteration.  Any output may be NULL.
 * No counterpart in the reference (it has no derivatives). */
int scft_diblock_stress(scft_diblock_t d, double dlnQ_dL[3], double* dF_dxN, double* Q_out);

/* Copy one stored propagator slice of the last iteration to host (as FP64): chain 0 is
 * q (slot u: qA(u) for u <= NsA, qB(u-NsA) after), chain 1 is q+ (qcA(u), then
 * qcB(u-NsA)); slot in [0, NsA+NsB].  The reference's qA/qB/qcA/qcB arrays
 * (src/crysSCFT_sample.cpp:457-460) hold the same values. */
int scft_diblock_get_contour(scft_diblock_t d, int chain, size_t slot, double* out);

/* Device pointers of the resident fields (space_size_phy FP64 each); any out may be NULL. */
int scft_diblock_device_fields(scft_diblock_t d, double** phiA, double** phiB, double** wA,
                               double** wB);

/* n_iter iterations on device-resident fields.  Per iteration i the host arrays (each may
 * be NULL) receive F[i], parts[4*i+0..3] = (enthalpic, -ln Q, entropic, xi term) as
 * print_energy forms them (src/crysSCFT_sample.cpp:404-418), maxinc[i] and Q[i].
 * Returns SCFT_ERR_NUMERIC if Q <= 0 or a NaN/Inf shows up. */
int scft_diblock_iterate(scft_diblock_t d, size_t n_iter, double* F, double* parts,
                         double* maxinc, double* Q);

/* End-to-end form for callers that keep fields in host memory: copies wA/wB in, runs
 * n_iter iterations, copies phiA/phiB and the updated wA/wB (in place) back out, with one
 * host synchronisation per call (page-locked wA/wB/phiA/phiB make the copies
 * asynchronous).  F, parts, maxinc, Q as in scft_diblock_iterate.  If an error code is
 * returned, phiA/phiB/wA/wB may already hold the values of the failed iteration. */
int scft_diblock_iterate_host(scft_diblock_t d, double* wA, double* wB, size_t n_iter,
                              double* phiA, double* phiB, double* F, double* parts,
                              double* maxinc, double* Q);

/* Arithmetic of the contour chains for the following iterations: SCFT_FP64 (the plain
 * form) or SCFT_FP32 (FP32 triplets on the tensor cores as 3xTF32 split products; Q,
 * phi, the free energy and the mixing stay FP64).  The precision form runs most
 * iterations in FP32 and finishes with FP64 "polish" iterations.  No counterpart in
 * the reference (FP64 only).  Buffers of a precision are allocated on first use. */
int scft_diblock_set_precision(scft_diblock_t d, int precision);
int scft_diblock_get_precision(scft_diblock_t d, int* out);

/* Field mixing of the iteration.  history = 0: the reference's simple mixing
 * w += acceptance (xN phi_other + ksi - w) (calc_new_fields, src/crysSCFT_sample.cpp:362-371;
 * the default).  history = 1..32: Anderson mixing over the last `history` iterates with
 * mixing parameter beta > 0, entirely on the device (no counterpart in the reference):
 * with residual r = (xN phiB + ksi - wA, xN phiA + ksi - wB) and D_j = r_0 - r_j it solves
 * sum_j <D_i, D_j> c_j = <D_i, r_0> and sets w <- w_0 + sum_j c_j (w_j - w_0)
 * + beta (r_0 + sum_j c_j (r_j - r_0)); a singular system restarts the history.
 * The history is cleared by this call and by scft_diblock_set_fields. */
int scft_diblock_set_mixing(scft_diblock_t d, int history, double beta);

/* Poll limit of every bounded wait inside the contour kernels (release flags, grid
 * barriers, tile loads; default 20,000,000, about a second).  A wait that runs out makes
 * the kernel record an error, let its own copies land and return, and the iteration call
 * returns SCFT_ERR_TIMEOUT; the context stays usable.  No counterpart in the reference
 * (it has no device code); a small limit is how the timeout path is tested. */
int scft_diblock_set_wait_limit(scft_diblock_t d, long long spins);

/* Where the FP64 iterations integrate phi_A and phi_B over the contour (integrate_phi,
 * src/crysSCFT_sample.cpp:348-360, trapezoid weights): fused = 1 (default) lets the
 * whole-contour kernel on cubic grids add q(s) q+(s) tile by tile as the second chain
 * reaches each slot, so a short kernel finishes phi instead of a pass over the stored
 * contour; fused = 0 always uses that separate pass.  The two agree to rounding (the sums
 * run in a different order).  The fused form applies to the alternating whole-contour
 * kernel with an even number of contour steps; other plans use the separate pass either
 * way.  No counterpart in the reference (a form switch of this library). */
int scft_diblock_set_phi_form(scft_diblock_t d, int fused);

/* rms residual sqrt(<r, r> / 2M) of each iteration of the last scft_diblock_iterate
 * call (any mixing); *count = number of iterations, at most `capacity` copied. */
int scft_diblock_get_residuals(scft_diblock_t d, double* out, size_t capacity, size_t* count);

/* Number of kernel launches the last scft_diblock_iterate issued per iteration. */
int scft_diblock_launches_per_iteration(scft_diblock_t d, size_t* out);

/* Phase timer, the GPU counterpart of the reference's std::clock() sum around
 * diffusion() (src/crysSCFT_sample.cpp:389-391): runs n_iter iterations without the
 * CUDA graph, with CUDA events between phases, and returns milliseconds per iteration:
 * out[0] whole iteration, out[1] the propagator chains (all triplets), out[2] Q + phi,
 * out[3] Boltzmann factors + energy + field update.  The fields advance as in iterate(). */
int scft_diblock_time_phases(scft_diblock_t d, size_t n_iter, double out[4]);

/* One triplet in place on a device buffer, like scft_solver_diffusion_device, but
 * allocating nothing: no cudaMalloc, cudaFree or allocating library call, ever.
 * No counterpart in the reference (its solvers allocate on the host in their
 * constructors).  It is for callers that cannot allocate device memory: programs
 * whose device memory is entirely owned by another framework's pool, and code paths
 * that must not call cudaMalloc/cudaFree because those calls can synchronise the
 * device.  The solver itself (operators) must have been set up beforehand.
 * Scratch: a static device array inside the library of
 * 2 x SCFT_STATIC_SCRATCH_MAX_POINTS doubles (4 MiB), held by every GPU that loads
 * the library until the process exits.  Solvers with space_size_phy above
 * SCFT_STATIC_SCRATCH_MAX_POINTS are rejected with SCFT_ERR_INVALID_ARG, and 3m
 * solvers whose triplet has several Kronecker terms with SCFT_ERR_UNSUPPORTED (both
 * before any device work).  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress), and so does the first call after that device's context
 * was replaced (cudaDeviceReset); make that first call before any stream capture.
 * All calls on a device share the
 * one array, so calls that overlap on the GPU (different streams, or different
 * host threads) race and corrupt each other's results: serialise them. */
#define SCFT_STATIC_SCRATCH_MAX_POINTS 262144
int scft_solver_diffusion_device_static_scratch(scft_solver_t solver, double* d_io, void* stream);

/* ========================================================================
 * Batching form: many independent AB-diblock instances (each with its own grid,
 * cell, fA and chiN; one solver kind, ds, mixing and precision for all) advanced
 * together; one batch iteration is one CUDA-graph launch in which the instances'
 * contour kernels run concurrently.  No counterpart in the reference (one instance
 * per program run).
 * ======================================================================== */

/* grid_log: 3 n logical sizes; cell: 3 n lengths; fA, xN: n values each. */
int scft_batch_create(int kind, size_t n, const size_t* grid_log, const double* cell, const double* fA,
                      const double* xN, double ds, double acceptance, int precision, int device,
                      scft_batch_t* out);
int scft_batch_destroy(scft_batch_t b);
int scft_batch_size(scft_batch_t b, size_t* n);
/* The iteration context of instance i (owned by the batch; do not destroy). */
int scft_batch_instance(scft_batch_t b, size_t i, scft_diblock_t* d);
int scft_batch_set_fields(scft_batch_t b, size_t i, const double* wA, const double* wB);
int scft_batch_get_fields(scft_batch_t b, size_t i, double* phiA, double* phiB, double* wA, double* wB);
/* n_iter iterations of every instance; F and maxinc (may be NULL) get n_iter x n values,
 * iteration-major. */
int scft_batch_iterate(scft_batch_t b, size_t n_iter, double* F, double* maxinc);
/* Worker streams and contour-kernel form (0 automatic, 1 alternating layout, 2 two-phase,
 * 3 per-axis kernels, 4 one persistent launch: the contours of every FP64 instance whose
 * own plan is the alternating kernel run together in one cooperative launch, each chain
 * on a team of CTAs that own several x-planes / y-slabs each; the other instances keep
 * their own kernels).  Forms 0-3 launch one contour kernel per instance. */
int scft_batch_configure(scft_batch_t b, size_t nstreams, int form);
/* Form 4: fixed team sizes for the listed grid sides (sizes[i] must divide sides[i]);
 * chains of other sides get the planner's choice (scft_team_schedule).  count 0 clears
 * the table. */
int scft_batch_set_team_sizes(scft_batch_t b, size_t count, const int* sides, const int* sizes);
/* The form-4 plan of the current configuration (built if needed): CTAs of the launch (0 if
 * no instance runs in it), team tasks, instances in the launch, and the planned makespan
 * and the lower bound (team work / CTAs) in microseconds per iteration under the cost
 * model.  No counterpart in the reference. */
int scft_batch_team_plan(scft_batch_t b, int* grid, size_t* ntasks, size_t* ninstances, double* planned_us,
                         double* bound_us);
/* The form-4 planner on the host alone (no GPU): nchains chains with grid side n[j] and
 * U[j] contour steps on G CTAs; nfixed grid sides with team sizes fixed by the caller
 * (may be 0).  Chains of one grid side form a class; for a target makespan a class with
 * team size T runs in columns of T CTAs with its chains stacked in them, and takes the T
 * that needs fewest CTAs; the smallest target whose classes fit in G CTAs is kept.
 * size[j] receives each chain's team size; the tasks
 * (chain, rank in team, team size), grouped by CTA, go to task_chain/task_rank/task_size
 * (room for cap), CTA b's tasks being [task_begin[b], task_begin[b + 1]) (G + 1 entries);
 * *ntasks receives the count (also when cap is too small, which returns
 * SCFT_ERR_INVALID_ARG).  planned_us / bound_us: makespan and its lower bound per
 * iteration under the planner's cost model.  No counterpart in the reference. */
int scft_team_schedule(size_t nchains, const int* n, const int* U, int G, size_t nfixed, const int* fixed_sides,
                       const int* fixed_sizes, int* size, size_t cap, int* task_chain, int* task_rank,
                       int* task_size, int* task_begin, size_t* ntasks, double* planned_us, double* bound_us);
/* Kernel launches of one batch iteration in the current configuration. */
int scft_batch_launches_per_iteration(scft_batch_t b, size_t* n);
/* Time n_trial batch iterations for each candidate configuration, keep the fastest.
 * The fields of every instance are restored afterwards (also when a trial fails; then the
 * configuration the batch had before the call is restored too).  Restoring the fields
 * goes through scft_batch_set_fields, so it clears each instance's Anderson mixing
 * history, as scft_diblock_set_fields does. */
int scft_batch_autotune(scft_batch_t b, size_t n_trial, size_t* best_nstreams, int* best_form, double* best_ms);

/* Measured FP64 throughput of `device` in TFLOP/s: FMA on the CUDA cores and
 * m8n8k4 MMA on the tensor cores (the denominator of the FP64 roofline).  No
 * counterpart in the reference (it has no GPU path). */
int scft_measure_fp64_peak(int device, double* tflops_simt, double* tflops_tensor);

/* Make the solver (and every diblock built on it) issue its work on `stream`
 * (a cudaStream_t; NULL restores the solver's own stream). */
int scft_solver_set_stream(scft_solver_t solver, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CRYSSCFT_B200_H */
