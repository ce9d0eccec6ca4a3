/*
 * hirensi_b200.h -- C ABI of the B200 (sm_100a) implementation of HiReNSI's
 * explicit 3D elastic forward / adjoint / gradient time loop.
 *
 * Plain C types only.  Every entry returns 0 on success or an HRN_E* code;
 * hrn_last_error() gives the message.  Host arrays are read or written
 * synchronously; the context owns all device memory.  A context is used by one
 * host thread at a time.
 *
 * Array conventions (C row-major, 0-based unless stated):
 *   CSR operators: PETSc AIJ layout (MatGetRowIJ / MatSeqAIJGetArray), 0-based,
 *                  columns sorted within each row.
 *   xyz[nj][3], inod[nel][27] (SHAPE_3_27 local order), id[nj][9] equation
 *   numbers with -1 for a constrained DOF, pml_param[6][4].
 *   u_store[nstep+1][nstore]   == Fortran U_Store_Mapping(NStore, 0:NStep)
 *   dis_meas[nshot][nrec3][nstep+1]; per shot == Fortran Dis_meas(0:NStep, NNDH*3)
 *
 * Each entry names the reference routine it replaces (file:line inside the
 * HiReNSI project, S4 = step_4_3D_Forward_and_Inverse).
 */
#ifndef HIRENSI_B200_H
#define HIRENSI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HRN_OK 0
#define HRN_EARG 1      /* invalid argument or size */
#define HRN_ECUDA 2     /* CUDA runtime error */
#define HRN_EOOM 3      /* device allocation failed */
#define HRN_ESTATE 4    /* entry called before its prerequisites */
#define HRN_ENAN 5      /* non-finite value detected in a reduction */
#define HRN_EMESH 6     /* non-positive Jacobian, top PML zone or bad face load */

#define HRN_FP64 0      /* stepping in FP64 */
#define HRN_FP32 1      /* stepping in FP32, FP64 reductions */

#define HRN_MAX_SHOTS 8 /* shots advanced together in one pass over the operator */

typedef struct hrn_ctx hrn_ctx;

/* Library version (major * 10000 + minor * 100 + patch). */
int hrn_version(void);

/* Create a context on CUDA device `device` with stepping precision HRN_FP64 or HRN_FP32. */
int hrn_create(int device, int precision, hrn_ctx **out);
int hrn_destroy(hrn_ctx *ctx);
const char *hrn_last_error(const hrn_ctx *ctx);

/* ---- operator ------------------------------------------------------------- */

/* Drop-in for the assembled PETSc matrices AC, AK, AG and the vector DIAG_M that
 * S4/Solve_Forward.F90:14-97 hands to EXPLICIT_RK4_PETSC_PML_3D.  Matrices are
 * passed unscaled; the library applies -M^-1 (forward, S4/Solver_PETSc_Explicit.F90:815-824)
 * and M (.) M^-1 (adjoint, :1222-1229) itself and never mutates caller data. */
int hrn_set_operator_csr(hrn_ctx *ctx, int32_t neq,
                         const int32_t *c_ia, const int32_t *c_ja, const double *c_a,
                         const int32_t *k_ia, const int32_t *k_ja, const double *k_a,
                         const int32_t *g_ia, const int32_t *g_ja, const double *g_a,
                         const double *diag_m);

/* Mesh for device assembly and for the gradient (the XYZ, INOD, MTEL, ID and
 * PML_PARAM arguments of ASSEM_*_PETSC_3D and of ..._Control_OtD). */
int hrn_set_mesh(hrn_ctx *ctx, int32_t nj, int32_t nel, int32_t neq,
                 const double *xyz, const int32_t *inod, const int32_t *mtel,
                 const int32_t *id, const double *rho_el, const double *pml_param);

/* Operator mode, chosen after hrn_set_mesh and before the first assembly.
 * matrix_free_only = 0 (default): hrn_assemble builds the CSR of C, K, G as below, and
 * every stage variant is available.  matrix_free_only = 1: hrn_assemble computes only
 * DIAG_M, and C, K, G are applied element by element from the mesh and the nodal
 * material (variants 90-95 / 100-105).  This needs no stored entries, so meshes whose
 * CSR would not fit the device (or the 2^31 entry range) can run.  No reference
 * counterpart: the reference always assembles PETSc matrices. */
int hrn_set_operator_mode(hrn_ctx *ctx, int32_t matrix_free_only);

/* Device assembly of C, K, G and DIAG_M from nodal lambda, mu (host arrays [nj]):
 * replaces ASSEM_REGULAR_DOMAIN_PETSC_3D (S4/Assemble_PETSc_3D.F90:6-184) and
 * ASSEM_PML_PETSC_3D (:192-436).  The first call fixes the sparsity pattern
 * (entries with a nonzero element contribution, as MAT_IGNORE_ZERO_ENTRIES). */
int hrn_assemble(hrn_ctx *ctx, const double *lambda, const double *mu);

/* hrn_assemble with lambda, mu already on the device (device pointers [nj]). */
int hrn_assemble_device(hrn_ctx *ctx, const double *d_lambda, const double *d_mu);

/* Download the current operator (unscaled).  With ia/ja/a NULL only *nnz is set
 * (0 for a matrix-free operator, which has no entries to download). */
int hrn_get_operator_csr(hrn_ctx *ctx, int32_t which, int32_t *ia, int32_t *ja, double *a, int64_t *nnz);
int hrn_get_diag_m(hrn_ctx *ctx, double *diag_m);

/* One per-step operator of the time loops applied to a host vector x [neq]:
 * adjoint = 0: y = -iM A x, the scaled matrix of EXPLICIT_RK4_PETSC_PML_3D
 * (S4/Solver_PETSc_Explicit.F90:815-824); adjoint = 1: y = A'^T x with A' the
 * adjoint-scaled matrix applied by MatMultTransposeAdd in the adjoint
 * (:1219-1229, 1319-1364).  which: 0 = C, 1 = K, 2 = G.  It reads the device
 * values the stage kernels stream, so dot-product tests can check the device
 * operator.  Not available for a matrix-free operator (HRN_ESTATE). */
int hrn_apply_operator(hrn_ctx *ctx, int32_t which, int32_t adjoint, const double *x, double *y);

/* Face-traction force vector B of ASSEM_FORCE_PETSC_3D (S4/Assemble_PETSc_3D.F90:444-548)
 * with ELEMENT_FS_3D (S4/Element_Matrices_3D.F90:890-1096), built on the device: a unit
 * vertical traction (Tx = Ty = 0, Tz = 1) integrated with the 3-point GLL rule over the
 * loaded face of every regular-domain element.  nface[nel] = ID_BC(IEL, 1): 0 = no load,
 * 1..6 = the loaded face (6 is taken as 5, as in the reference).  A face point off the
 * surface (|z| > 1e-3) returns HRN_EMESH, where the reference STOPs.  B stays on the
 * device for hrn_set_shots_face_force; b [neq] (may be NULL) receives a host copy. */
int hrn_assemble_face_force(hrn_ctx *ctx, const int32_t *nface, double *b);

/* hrn_set_shots with the device face-force vector of hrn_assemble_face_force as the B of
 * every shot (the B argument of EXPLICIT_RK4_PETSC_PML_3D, S4/Solve_Forward.F90:117-119),
 * each scaled by its own TIME_FUNCTION table ftab[nshot][nstep+1][3]. */
int hrn_set_shots_face_force(hrn_ctx *ctx, int32_t nshot, int32_t nstep, double dt, const double *ftab);

/* ---- problem description --------------------------------------------------- */

/* History equations U_Store_Numbers_Global (S3/PIC_Inversion_Data_Structure.F90:255-300). */
int hrn_set_history(hrn_ctx *ctx, int32_t nstore, const int32_t *store_eq);

/* Shots advanced together.  Source = nsrc entries of the unscaled force vector B
 * per shot (src_b[nsrc][nshot], zero where a shot has no load at that equation),
 * scaled by TIME_FUNCTION samples ftab[nshot][nstep+1][3] at T, T+dt, T+dt/2
 * (S4/Solver_PETSc_Explicit.F90:983-995). */
int hrn_set_shots(hrn_ctx *ctx, int32_t nshot, int32_t nstep, double dt,
                  int32_t nsrc, const int32_t *src_eq, const double *src_b, const double *ftab);

/* Receivers: EqDis (equations) and EqDis_MAP_U_Store_Numbers_Global (0-based
 * positions in the history), S4/IO_Parallel_Inversion.F90:116-133. */
int hrn_set_receivers(hrn_ctx *ctx, int32_t nrec3, const int32_t *eqdis, const int32_t *eqdis_map);

/* Shots of uneven record length and receiver count advanced in one batch.  The
 * reference runs one source per solve, with its own NSTEP and EqDis
 * (S4/Solver_PETSc_Explicit.F90:660-1405, S4/Solver_PETSc_Inverse.F90:591-657); here
 * shot s records steps 0..nstep_shot[s] (1 <= nstep_shot[s] <= nstep of
 * hrn_set_shots), and receiver entry q of hrn_set_receivers belongs to it when
 * rec_mask[s * nrec3 + q] != 0.  Its misfit counts steps 1..nstep_shot[s] and its
 * receivers only, and its adjoint starts at its own last step, so every shot's
 * misfit, traces and gradient share equal those of the shot solved alone.  The
 * batch still steps nstep times, and the forward history past a shot's length is
 * computed but unused.  NULL leaves all shots at nstep / every receiver.  Reset by
 * hrn_set_shots (both) and hrn_set_receivers (the mask). */
int hrn_set_shot_records(hrn_ctx *ctx, const int32_t *nstep_shot, const uint8_t *rec_mask);

/* Measured data Dis_meas of every shot, kept on the device for hrn_misfit and
 * hrn_adjoint_gradient called with dis_meas = NULL (on_device: dis_meas is a
 * device pointer).  Replaces the measured-data read of
 * Input_Inv_Measured_Data (S4/PTC_Input.F90:961-1046). */
int hrn_set_data(hrn_ctx *ctx, const double *dis_meas, int32_t on_device);

/* ---- time loops ------------------------------------------------------------ */

/* Forward-wavefield checkpointing for the adjoint.  interval 0 (the default)
 * keeps the whole history U_Store(NStore, 0:NSTEP) on the device, as the
 * reference does.  interval K > 0 keeps instead the forward state every K steps
 * and the receiver displacements of every step.  hrn_adjoint_gradient then
 * recomputes the history of each K-step segment from its checkpoint before
 * stepping the adjoint through it.  This costs one more forward pass and needs
 * device memory for about (NSTEP/K) states + K history rows.  With
 * checkpointing, hrn_get_history is unavailable; misfit, traces and gradient
 * are the same. */
int hrn_set_checkpointing(hrn_ctx *ctx, int32_t interval);

/* Forward RK4 for all shots, EXPLICIT_RK4_PETSC_PML_3D (S4/Solver_PETSc_Explicit.F90:660-1117).
 * The history U_Store of every shot stays on the device. */
int hrn_forward(hrn_ctx *ctx);
int hrn_get_history(hrn_ctx *ctx, int32_t shot, double *u_store);
/* Receiver traces U_Store(EqDis_MAP, 0:NStep) of every shot: traces[nshot][nrec3][nstep+1]. */
int hrn_get_traces(hrn_ctx *ctx, double *traces);

/* Full forward state of one shot at a checkpointed step (step a multiple of the
 * checkpoint interval, 0 <= step <= NSTEP): x1 (time integral of u), x2 = u and
 * x3 = du/dt over all equations, [neq] each; NULL skips an array.  This is the
 * data of the reference's ParaView snapshots, which scatter x2 of every
 * NSParaview-th step to the nodes (S4/Solver_PETSc_Explicit.F90:936-975,
 * S4/ParaView.F90:1206-1440); hirensi_b200/snapshots.py writes the files. */
int hrn_get_state(hrn_ctx *ctx, int32_t step, int32_t shot, double *x1, double *x2, double *x3);

/* Compute_Misfit (S4/Solver_PETSc_Inverse.F90:591-657) summed over shots;
 * dis_meas NULL uses the data of hrn_set_data. */
int hrn_misfit(hrn_ctx *ctx, const double *dis_meas, double *cost);

/* The misfit of hrn_misfit for callers that cannot allocate device memory.
 * It has no counterpart in the reference.  d_dis_meas is a DEVICE pointer to
 * Dis_meas laid out as for hrn_set_data ([nshot][nrec3][nstep+1]); it is read
 * in place and not kept.  A host pointer, or memory of another device, returns
 * HRN_EARG before anything is launched.  The scratch is one static device array
 * shared by every context and call in the process, so nothing is allocated.
 * Limit: nshot * (nstep + 1) <= 131072, larger problems return HRN_EARG.  The
 * first call on a device does the set-up: it looks the array's address up
 * (cudaGetSymbolAddress) with that device current and keeps it, so make that first
 * call before any stream capture begins, and do not use the entry across a
 * cudaDeviceReset.  Calls whose kernels overlap on one GPU (other streams, other
 * contexts, other host threads) race on the scratch: serialize them.  It
 * synchronizes its stream and returns once *cost is ready. */
int hrn_misfit_noalloc(hrn_ctx *ctx, const double *d_dis_meas, double *cost);

/* Adjoint RK4 (OtD) with the zero-lag gradient fused into each step:
 * EXPLICIT_RK4_PETSC_PML_3D_Adjoint_OtD (:1125-1405) followed by
 * EXPLICIT_RK4_PETSC_PML_3D_Control_OtD (:1413-1522), summed over shots.
 * g_lambda, g_mu [nj] receive the raw accumulated gradient (before the sign
 * flip and mass scaling of S4/Program_Main.F90:412-455).  lambda_2mu selects
 * ELEMENT_g_3D_v2.  keep_p stores the adjoint history for hrn_get_adjoint_history.
 * dis_meas NULL uses the data of hrn_set_data; g_lambda / g_mu NULL leave the
 * gradient on the device (hrn_get_gradient_device). */
int hrn_adjoint_gradient(hrn_ctx *ctx, const double *dis_meas, int32_t lambda_2mu, int32_t keep_p,
                         double *g_lambda, double *g_mu);
int hrn_get_adjoint_history(hrn_ctx *ctx, int32_t shot, double *p_store);
/* Copy the accumulated gradient to device buffers [nj] (either may be NULL). */
int hrn_get_gradient_device(hrn_ctx *ctx, double *d_g_lambda, double *d_g_mu);

/* ---- model update of the inversion loop (device vectors, FP64) ------------------
 * All vector arguments are device pointers of length n (nodal vectors: n = nj).
 * Reductions are deterministic (fixed-order two-pass sums). */

/* out = x . y  (VecDot) */
int hrn_vec_dot(hrn_ctx *ctx, int32_t n, const double *x, const double *y, double *out);
/* kind 2: Euclidean norm, kind 0: max norm (VecNorm NORM_2 / NORM_INFINITY) */
int hrn_vec_norm(hrn_ctx *ctx, int32_t n, const double *x, int32_t kind, double *out);
/* z = a x + b y (y may be NULL: z = a x); covers VecAXPY, VecWAXPY, VecScale, VecCopy */
int hrn_vec_axpby(hrn_ctx *ctx, int32_t n, double a, const double *x, double b, const double *y, double *z);
/* z = x .* y (VecPointwiseMult) */
int hrn_vec_mul(hrn_ctx *ctx, int32_t n, const double *x, const double *y, double *z);
/* x = min(max(x, lo), hi): the material bounds of S4/Program_Main.F90:651-678 */
int hrn_vec_clip(hrn_ctx *ctx, int32_t n, double lo, double hi, double *x);
/* y[i] = x[map[i]]: the PML material extension scatter (vscat_mat_extend, :633-636) */
int hrn_vec_gather(hrn_ctx *ctx, int32_t n, const int32_t *map, const double *x, double *y);

/* TV regularization vectors and costs of the nodal lambda, mu
 * (Assem_TV_TN_Regularization, S4/Assemble_PETSc_3D.F90:755-849, unweighted). */
int hrn_regularization_tv(hrn_ctx *ctx, const double *d_lambda, const double *d_mu, double *d_reg_lambda,
                          double *d_reg_mu, double *cost_lambda, double *cost_mu);
/* Lumped gradient mass Mg per node (Assem_R_Mg_3D, S4/Assemble_PETSc_3D.F90:670-747). */
int hrn_gradient_mass(hrn_ctx *ctx, double *d_mg);

/* Coupled L-BFGS with memory m (S4/LBFGS_Coupled.F90).  restriction[nj] is 1 in
 * the regular domain, 0 in the PML (S4/Control_Problem_Operators.F90:14-22). */
int hrn_lbfgs_setup(hrn_ctx *ctx, int32_t m, const double *d_restriction);
/* p = -H g for iteration `iter` (p = -g when iter == iter_begin); rho_out gets
 * 1 / (y_lambda.s_lambda + y_mu.s_mu) of the new pair (may be NULL). */
int hrn_lbfgs_direction(hrn_ctx *ctx, int32_t iter, int32_t iter_begin, const double *g_lambda, const double *g_mu,
                        const double *g_lambda_pre, const double *g_mu_pre, const double *lambda, const double *mu,
                        const double *lambda_pre, const double *mu_pre, double *p_lambda, double *p_mu, double *rho_out);

/* ---- streams and timing -------------------------------------------------------- */

/* Launch all work of this context on `stream` (a cudaStream_t, NULL = the
 * context's own stream).  The caller keeps the stream alive. */
int hrn_set_stream(hrn_ctx *ctx, void *stream);

/* CUDA graphs of the time loops (on by default).  hrn_forward and
 * hrn_adjoint_gradient capture all launches of a call -- every stage, source,
 * history, trace and gradient launch of every step -- into one graph on the
 * context's stream and replay it on later calls while no setting has changed and
 * no buffer of the context has been reallocated; new values in the buffers (a
 * reassembled operator, new data) need no new capture.  Calls with timing on, on
 * the legacy default stream, or the first call of a variant still to be tuned run
 * the launches directly.  No reference counterpart: the reference steps with
 * PETSc calls from the host. */
int hrn_set_graphs(hrn_ctx *ctx, int32_t enable);

/* Time loops captured and graph launches made by this context so far. */
int hrn_graph_stats(hrn_ctx *ctx, int64_t *captures, int64_t *replays);

/* With timing on, every launch of the fused RK4 stage kernel is bracketed by
 * CUDA events on the launching stream. */
int hrn_set_timing(hrn_ctx *ctx, int32_t enable);

/* Device time of the last hrn_forward / hrn_adjoint_gradient, and the summed
 * duration and number of launches of the fused stage kernel since timing was
 * last enabled. */
int hrn_last_timing(hrn_ctx *ctx, double *total_ms, double *stage_kernel_ms, int64_t *stage_launches);

/* Device time of one stage launch alone: nsteps RK4 steps (4 stage launches each)
 * of the tuned variant of the forward (adjoint = 0) or adjoint operator, launched
 * back to back from a zeroed state with the first step's sources and no history,
 * bracketed by one pair of CUDA events on the context's stream;
 * *avg_stage_ms = elapsed / (4 nsteps).  The forward history stays valid; the
 * state buffers are overwritten.  Needs a tuned variant (after hrn_forward /
 * hrn_adjoint_gradient).  No reference counterpart: a measurement aid. */
int hrn_time_stage(hrn_ctx *ctx, int32_t adjoint, int32_t nsteps, double *avg_stage_ms);

/* Stage-kernel variant per operator (forward, adjoint): lanes per row * 10 +
 * (1 if the stage inputs are materialized by the previous stage, 0 if rebuilt
 * at every gather) + (2 for the tiled kernel that stages the matrix slab of
 * each tile in shared memory with bulk copies, 4 for the kernel over compact
 * row tiles that stages each tile's distinct gathered records in shared
 * memory); lanes in {4, 8, 16}, tiled with 4 or 8.  90-95 / 100-105: the
 * matrix-free element kernels (operator assembled from the mesh).  0 = time all
 * variants on first use and keep the fastest (the default after every new
 * sparsity pattern). */
int hrn_set_variant(hrn_ctx *ctx, int32_t forward, int32_t adjoint);
int hrn_get_variant(hrn_ctx *ctx, int32_t *forward, int32_t *adjoint);

/* Number of kernels this context has launched since it was created. */
int hrn_launch_count(hrn_ctx *ctx, int64_t *n);

/* ---- learned gradient preconditioner ---------------------------------------
 * No counterpart in the reference.  The inversion can ask a small 3-D CNN for a
 * positive diagonal scale of the gradient; the line search on the true misfit
 * accepts the scaled direction or falls back to L-BFGS. */

/* Source illumination of every stored node: sum over steps, shots and x, y, z of
 * u^2 from the forward history.  d_out: device array [nstore / 3], in the order of
 * the history rows (needs the whole history, i.e. no checkpointing). */
int hrn_illumination(hrn_ctx *ctx, double *d_out);

/* Diagonal pseudo-Hessian of the lambda / mu model from the forward history: the
 * zero-lag correlation of the gradient (..._Control_OtD, S4/Element_Matrices_3D.F90:
 * 1725-1890) with the forward wavefield in place of the adjoint one, i.e.
 * dt * sum_n sum_shots of (div u)^2 (lambda) and of the strain-energy term (mu),
 * n = 1 .. NSTEP-1, at the regular-domain nodes.  d_h_lambda, d_h_mu: device
 * arrays [nj], overwritten.  Needs the whole forward history. */
int hrn_pseudo_hessian(hrn_ctx *ctx, double *d_h_lambda, double *d_h_mu);

/* 3x3x3 convolution with zero padding on the 5th-generation tensor cores (tcgen05.mma,
 * BF16 operands, FP32 accumulation in tensor memory): y = act(b + w * x), act = ReLU
 * when relu != 0.  Activations are channels-last with a channel stride of 16:
 * x [nz][ny][nx][16] BF16 with channels >= cin zero, y [nz][ny][nx][16] BF16 with
 * channels >= cout written as zero.  w is [cout][cin][27] BF16 (tap k = 9 dz + 3 dy + dx),
 * bias [cout] FP32.  At most 16 channels in and out; (nz + 2)(ny + 2)(nx + 2) at most
 * 2^30.  All pointers are device pointers; stream is a cudaStream_t or NULL.  Returns
 * once the layer has run (the kernels' error flag is read back).  The layers keep a
 * per-device scratch (the packed weights, a copy of the input with a one-voxel zero
 * border, weight-gradient partial sums), allocated when a larger grid first needs it
 * and shared by all calls on that device: calls that overlap on one device race on it. */
int hrn_cnn_conv3d_forward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                           const void *w, const float *bias, int32_t relu, void *y, void *stream);
/* Gradients of that layer from gy = dL/dy (FP32 [nz][ny][nx][16]): gx = dL/dx (FP32
 * [nz][ny][nx][16], channels >= cin zero; skipped when NULL), gw = dL/dw [cout][cin][27]
 * and gb = dL/db [cout] (FP32, overwritten).  y is the forward output (for the ReLU mask).
 * The masked gy is rounded to BF16 as the tensor-core operand of gx and gw; gb sums it in
 * FP32.  Partial sums over voxel chunks are added in a fixed order. */
int hrn_cnn_conv3d_backward(int32_t cin, int32_t cout, int32_t nz, int32_t ny, int32_t nx, const void *x,
                            const void *w, const void *y, int32_t relu, const float *gy, float *gx, float *gw,
                            float *gb, void *stream);

#ifdef __cplusplus
}
#endif
#endif
