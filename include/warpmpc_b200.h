/*
 * warpmpc_b200.h -- C ABI of the B200-native batched fixed-pattern
 * QDLDL (LDL^T) / OSQP-ADMM library (libwarpmpc_b200.so, sm_100a).
 *
 * Every entry point returns an int status (WMPC_OK = 0) and never throws.
 * wmpc_last_error_string() returns a thread-local message for the last
 * failure on the calling thread.  All device pointers are caller-owned
 * (inputs, outputs and workspace); a plan owns only its uploaded pattern
 * tables.  Compute entry points are stream-ordered and launch-only: they
 * allocate nothing and do not synchronize the host.
 *
 * Layouts.  "Symbolic-major" arrays hold element (i, b) at [i * ld + b]
 * (rows = KKT / L / value index, columns = instance b), exactly the
 * (nnz, batch) / (n, batch) layout of the reference's Warp backend
 * (values_layout="original_symbolic", rhs_layout="symbolic",
 * warpmpc/jax_qdldl/warp_backend.py:1302-1408).  A "batch stride" of 0
 * broadcasts one instance over the batch.  "Batch-major" arrays hold
 * (b, i) at [b * ld + i], the layout of the reference's OSQP API
 * (warpmpc/jax_osqp/solver.py:934-982).
 *
 * Floating point: float32 throughout, the reference's operation order with
 * separately rounded products and sums (no multiply-add contraction).
 */
#ifndef WARPMPC_B200_H
#define WARPMPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* wmpc_stream_t; /* cudaStream_t */

enum {
  WMPC_OK = 0,
  WMPC_ERR_INVALID_ARGUMENT = 1,
  WMPC_ERR_CUDA = 2,
  WMPC_ERR_UNSUPPORTED = 3,
  WMPC_ERR_WORKSPACE = 4,
  WMPC_ERR_OUT_OF_MEMORY = 5
};

/* Per-instance status words written by the OSQP entry points. */
enum {
  WMPC_STATUS_MAX_ITER = 0,      /* ran max_iter iterations (reference behaviour) */
  WMPC_STATUS_SOLVED = 1,        /* met the eps_abs/eps_rel termination test */
  WMPC_STATUS_NONFINITE = 2,     /* a non-finite iterate or residual appeared */
  WMPC_STATUS_ZERO_PIVOT = 4,    /* D had an exact zero or non-finite pivot */
  WMPC_STATUS_KERNEL_ABORT = 8   /* a device pipeline wait timed out; results invalid */
};

/* ------------------------------------------------------------------ */
/* Pattern (QDLDL plan) tables, host pointers, int32.                  */
/* Produced by the host planner (build_qdldl_plan), ragged form of      */
/* QDLDLPlan: warpmpc/jax_qdldl/types.py:11-53, core.py:147-256.        */
/* ------------------------------------------------------------------ */
typedef struct wmpc_pattern_desc {
  int32_t n;       /* KKT dimension                                   */
  int32_t nnz_a;   /* stored upper-triangle entries (original order)  */
  int32_t nnz_l;   /* strictly-lower entries of L                     */
  const int32_t* perm_to_orig; /* [nnz_a] permuted slot -> original slot */
  const int32_t* diag_pos;     /* [n] permuted slot of diagonal k        */
  const int32_t* init_ptr;     /* [n+1] off-diagonal entries of column k */
  const int32_t* init_rows;    /* [init_ptr[n]]                          */
  const int32_t* init_pos;     /* [init_ptr[n]] permuted slots           */
  const int32_t* proc_ptr;     /* [n+1] row program of row k             */
  const int32_t* proc_cols;    /* [nnz_l] column cidx visited            */
  const int32_t* proc_lidx;    /* [nnz_l] L slot written                 */
  const int32_t* proc_offsets; /* [nnz_l] entries of cidx already set    */
  const int32_t* lp;           /* [n+1] CSC column pointers of L         */
  const int32_t* li;           /* [nnz_l] CSC row indices of L           */
  const int32_t* p;            /* [n] permutation (new -> old)           */
  const int32_t* pinv;         /* [n] inverse permutation                */
} wmpc_pattern_desc;

typedef struct wmpc_plan wmpc_plan;

/* Upload a pattern to `device`.  Replaces the host plan the reference
 * builds in build_qdldl_plan (warpmpc/jax_qdldl/core.py:259-311) and the
 * jnp.asarray uploads of compile_qdldl_warp (warp_backend.py:1230-1286). */
int wmpc_plan_create(const wmpc_pattern_desc* desc, int device, wmpc_plan** out);
int wmpc_plan_destroy(wmpc_plan* plan);
/* Number of int32 table entries resident on the device (diagnostics). */
int wmpc_plan_info(const wmpc_plan* plan, int32_t* n, int32_t* nnz_a, int32_t* nnz_l,
                   int32_t* max_row_nnz, int32_t* max_col_nnz);

/* ------------------------------------------------------------------ */
/* Batched LDL^T factor / solve.                                       */
/* ------------------------------------------------------------------ */

/* Bytes of device workspace wmpc_factor / wmpc_solve / wmpc_factor_solve
 * need for `batch` instances (0 when the kernels stage everything in
 * shared memory). */
size_t wmpc_factor_workspace_bytes(const wmpc_plan* plan, int32_t batch);
size_t wmpc_solve_workspace_bytes(const wmpc_plan* plan, int32_t batch);

/* Numeric factorization.  Replaces CompiledQDLDL.factor of the Warp
 * backend (warp_backend.py:1302-1349 -> _qdldl_factor[_segmented]_transpose_kernel
 * 41-173).  values: [nnz_a x batch] symbolic-major, original (un-permuted)
 * upper-CSC order, batch stride values_bstride (0 = one shared matrix).
 * Outputs lx [nnz_l x batch], d, dinv [n x batch] (ld = batch). */
int wmpc_factor(const wmpc_plan* plan, const float* values, int64_t values_ld,
                int32_t values_bstride, float* lx, float* d, float* dinv, int32_t batch,
                void* workspace, size_t workspace_bytes, wmpc_stream_t stream);

/* Triangular solve x = P^T L^-T D^-1 L^-1 P rhs.  Replaces CompiledQDLDL.solve
 * (warp_backend.py:1351-1402 -> serial/segmented/level kernels 176-454).
 * lx [nnz_l x *], dinv [n x *] with batch stride factor_bstride (0 = one
 * factor shared by every right-hand side); rhs, x [n x batch] (ld = batch);
 * x may alias rhs. */
int wmpc_solve(const wmpc_plan* plan, const float* lx, const float* dinv,
               int32_t factor_bstride, const float* rhs, float* x, int32_t batch,
               void* workspace, size_t workspace_bytes, wmpc_stream_t stream);

/* Allocation-free variant of wmpc_solve (no counterpart in the reference).
 * For callers that cannot allocate device memory when they solve -- a
 * real-time control loop that must stay out of the CUDA allocator, or a
 * framework custom-call handler with no slot for an extra workspace: the
 * work vectors live in a fixed 32 MiB array of device memory inside this
 * library, so only inputs and outputs are passed.  Same arguments and
 * results as wmpc_solve.  Limit: n * batch <= 8,388,608 floats (larger
 * requests return WMPC_ERR_WORKSPACE and launch nothing).  All calls on a
 * device share the array: calls whose kernels may overlap on the GPU race
 * and must be ordered (same stream, or events).  The first call on a device
 * looks up the array's device address, so make it before any stream
 * capture that contains the call.  Allocates nothing. */
int wmpc_solve_noalloc(const wmpc_plan* plan, const float* lx, const float* dinv,
                       int32_t factor_bstride, const float* rhs, float* x, int32_t batch,
                       wmpc_stream_t stream);

/* factor then solve.  Replaces CompiledQDLDL.factor_and_solve
 * (warp_backend.py:1404-1408). */
int wmpc_factor_solve(const wmpc_plan* plan, const float* values, int64_t values_ld,
                      int32_t values_bstride, const float* rhs, float* x, float* lx, float* d,
                      float* dinv, int32_t batch, void* workspace, size_t workspace_bytes,
                      wmpc_stream_t stream);

/* ------------------------------------------------------------------ */
/* OSQP problem (FixedOSQPPlan: warpmpc/jax_osqp/types.py:86-132).     */
/* ------------------------------------------------------------------ */
typedef struct wmpc_osqp_desc {
  int32_t n;        /* variables                                      */
  int32_t m;        /* constraints                                    */
  int32_t nnz_p;    /* stored upper entries of P                      */
  int32_t nnz_a;    /* stored entries of A                            */
  int32_t nnz_kkt;  /* stored upper entries of the KKT matrix         */
  float sigma, alpha;
  const float* kkt_base;      /* [nnz_kkt] KKT values (fp32 of the plan's) */
  const int32_t* p_to_kkt;    /* [nnz_p]  */
  const float* p_diag_sigma;  /* [nnz_p]  */
  const int32_t* a_to_kkt;    /* [nnz_a]  */
  const float* p_scale;       /* [nnz_p]  */
  const float* a_scale;       /* [nnz_a]  */
  const int32_t* a_rows;      /* [nnz_a] CSC entry rows of A */
  const int32_t* a_cols;      /* [nnz_a] */
  const int32_t* p_full_rows; /* [nnz_pf] both triangles of P, reference order */
  const int32_t* p_full_cols;
  const int32_t* p_full_value_map;
  int32_t nnz_p_full;
  const float* rho_vec;       /* [m] */
  const float* rho_inv_vec;   /* [m] */
  const float* q_scale;       /* [n] c*D        */
  const float* scaling_d;     /* [n] D          */
  const float* scaling_dinv;  /* [n] 1/D        */
  const float* scaling_e;     /* [m] E          */
  const float* scaling_einv;  /* [m] 1/E        */
  const float* y_scale;       /* [m] c/E        */
  const float* y_unscale;     /* [m] E/c        */
  /* rho adaptation (optional; NULL disables it for this problem): each
   * constraint's rho class (-1 loose: rho_min, 0 inequality: rho,
   * 1 equality: 1e3 rho, as solver.py:164-183 assigns them), the KKT slot
   * of each constraint's -1/rho diagonal entry, and the plan's scalar rho. */
  const int32_t* rho_type;    /* [m] */
  const int32_t* rho_to_kkt;  /* [m] */
  float rho;
} wmpc_osqp_desc;

typedef struct wmpc_osqp wmpc_osqp;

/* Upload an OSQP problem bound to a KKT plan (same device). */
int wmpc_osqp_create(const wmpc_osqp_desc* desc, const wmpc_plan* kkt_plan, wmpc_osqp** out);
int wmpc_osqp_destroy(wmpc_osqp* osqp);

/* Solve options (OSQPSettings subset, warpmpc/jax_osqp/types.py:60-75). */
typedef struct wmpc_osqp_options {
  int32_t max_iter;
  int32_t check_termination; /* 0: exactly max_iter iterations (reference)  */
  float eps_abs, eps_rel;
  int32_t warm_start;        /* 1: x0/z0/y0 given (unscaled), 0: zeros       */
  int32_t reuse_factor;      /* 1: the workspace already holds the factor of
                                these P/A values from a previous call with the
                                same workspace, batch and mode: skip it       */
  int32_t adaptive_rho_interval; /* > 0: every this many iterations each
                                instance re-estimates its rho from its scaled
                                residuals (OSQP's rule, Stellato et al. 2020,
                                sec. 5.2) and, when the estimate is more than
                                adaptive_rho_tolerance times away, takes it and
                                refactors (plain mode; the reference has no
                                rho adaptation: solver.py:587-588) */
  float adaptive_rho_tolerance;
} wmpc_osqp_options;

/* Batched problem data, batch-major.  p_values [pb x nnz_p], a_values
 * [ab x nnz_a] with pb, ab in {1, batch}; q [batch x n]; l, u [batch x m];
 * warm start x0 [batch x n], z0, y0 [batch x m] (ignored unless
 * options.warm_start).  Outputs x [batch x n], z, y [batch x m],
 * prim_res, dual_res, obj [batch]; iters and status [batch] (int32, may be
 * NULL). */
typedef struct wmpc_osqp_batch {
  int32_t batch;
  const float* p_values; int32_t p_batch;
  const float* a_values; int32_t a_batch;
  const float* q; const float* l; const float* u;
  const float* x0; const float* z0; const float* y0;
  float* x; float* z; float* y;
  float* prim_res; float* dual_res; float* obj;
  int32_t* iters; int32_t* status;
  /* rho adaptation outputs (may be NULL): each instance's final scalar rho
   * and how many times it changed (one refactorization each) */
  float* rho; int32_t* rho_updates;
} wmpc_osqp_batch;

/* Device workspace bytes for `batch` instances.  mode: WMPC_OSQP_PLAIN or
 * WMPC_OSQP_PERSISTENT; external_factor: 1 when the caller passes lx/dinv
 * (solve_with_factor), 0 when the call factors. */
size_t wmpc_osqp_workspace_bytes(const wmpc_osqp* osqp, int32_t batch, int32_t mode, int32_t external_factor);

/* Which streaming schedule the problem carries (no reference counterpart: the
 * streaming kernel is this library's).  info[0]: 1 when persistent solves run
 * the streaming kernel's schedule, 0 when they fall back; info[1]: work-vector
 * slots of the frontier form that fixed-iteration solves of more 32-instance
 * tiles than SMs run (0: the plain form, one row per KKT index); info[2]: the
 * KKT dimension; info[3]: the frontier form's release lag.  The frontier form
 * is built when the problem is created with WMPC_STREAM_FRONTIER=1 (the only
 * schedule) or =2, the default (beside the plain one, used where it lets two
 * CTAs share an SM and the plain form does not); =0 builds only the plain
 * form. */
int wmpc_osqp_stream_info(const wmpc_osqp* osqp, int32_t info[4]);

enum { WMPC_OSQP_PLAIN = 0, WMPC_OSQP_PERSISTENT = 1 };

/* KKT assembly + numeric factorization.  Replaces CompiledOSQP.factor
 * (solver.py:799-804: assemble_kkt_values -> transpose -> qdldl.factor).
 * Factor batch fb = max(p_batch, a_batch); lx [nnz_l x fb], d, dinv
 * [n+m x fb] symbolic-major. */
int wmpc_osqp_factor(const wmpc_osqp* osqp, const float* p_values, int32_t p_batch, const float* a_values,
                     int32_t a_batch, float* lx, float* d, float* dinv, void* workspace,
                     size_t workspace_bytes, wmpc_stream_t stream);

/* mode WMPC_OSQP_PLAIN: the reference's loop structure with the CUDA
 * factor/solve as drop-in (solver.py:799-872: one factor, then max_iter x
 * {wmpc_solve, ADMM update + next right-hand side} as separate launches).
 * mode WMPC_OSQP_PERSISTENT: one fused launch per instance tile: KKT
 * assembly + factor + all ADMM iterations + residual epilogue, with an
 * optional termination test.  Replaces CompiledOSQP.solve /
 * solve_warm_start (solver.py:934-982).  When lx/dinv are non-NULL the
 * factorization is taken from them (factor_batch 1 = shared by all
 * instances, or batch): CompiledOSQP.solve_with_factor[_warm_start]
 * (solver.py:881-932). */
int wmpc_osqp_solve(const wmpc_osqp* osqp, const wmpc_osqp_options* options,
                    const wmpc_osqp_batch* data, const float* lx, const float* dinv,
                    int32_t factor_batch, int32_t mode, void* workspace, size_t workspace_bytes,
                    wmpc_stream_t stream);

/* Several problem classes (sparsity patterns) in one persistent launch: the
 * work-queue form of wmpc_osqp_solve(mode = WMPC_OSQP_PERSISTENT) for a
 * mixed-size batch (the reference solves each pattern with its own compiled
 * solver, solver.py:685-982; this walks every class's instance tiles in one
 * kernel, costliest class first, so classes of different sizes share the
 * GPU).  Per class i: osqps[i], options[i] (reuse_factor must be 0), data[i]
 * and its own workspace (workspaces[i], at least
 * wmpc_osqp_workspace_bytes(osqps[i], data[i].batch, WMPC_OSQP_PERSISTENT, 0)
 * bytes).  1 <= n_classes <= 6, all on one device.  Results as wmpc_osqp_solve,
 * per class; with options[i].check_termination > 0 an instance stops once its
 * largest unscaled iterate change over an iteration is at most eps_abs
 * (data[i].iters receives its iteration count; SOLVED in data[i].status comes
 * from the exact residuals of the returned iterate). */
int wmpc_osqp_solve_persistent(const wmpc_osqp* const* osqps, const wmpc_osqp_options* options,
                               const wmpc_osqp_batch* data, int32_t n_classes, void* const* workspaces,
                               const size_t* workspace_bytes, wmpc_stream_t stream);

/* Host-only export of the streaming schedule the persistent kernel uses for
 * a pattern (no counterpart in the reference; used to verify the schedule
 * on the CPU).  rho/rhoinv: per-constraint values (n_primal = number of
 * primal variables; KKT rows >= n_primal are constraints).  units/cols/rel:
 * backward chunk size targets (4-entry units, columns, releases); funits:
 * forward chunk target (units); offload: work also given to the releasing
 * warp (bit 0: leaf columns, bit 1: rows whose entries all read leaf rows);
 * bit 2 asks for the frontier-slot form (offload bits 0): the work vector
 * holds only the values a sweep still reads, in slots; right-hand sides and
 * forward results travel through the stages (what the streaming kernel runs
 * when a problem is created with WMPC_STREAM_FRONTIER=1); bits 8 and up, when
 * nonzero, set its release lag in chunks (default 4); bit 3 (with bit 2)
 * copies each row without entries from the stage into its slot at its
 * chunk's start instead of sweeping it as a unit.  With out == NULL, *out_words receives the
 * buffer size; otherwise out (capacity out_capacity int32 words) receives,
 * in order:
 *   [n_chunks, blen, max_units, max_cols, max_rel, max_meta_words, max_row_nnz, n_meta]
 *   chunk_off[n_chunks+1] chunk_units[n_chunks] chunk_cols[n_chunks]
 *   chunk_u0[n_chunks] chunk_nrel[n_chunks] meta_off[n_chunks] meta_words[n_chunks] meta[n_meta]
 *   col_uoff[n] dinv_off[n] proc_boff[nnz_l] u_perm[n] u_orig[n]
 *   init_slot[init_ptr[n]] upd_ptr[nnz_l+1] upd_slot[upd_ptr[nnz_l]]
 *   [n_fchunks, flen, max_funits, max_fmeta_words, n_fmeta]
 *   fchunk_off[n_fchunks+1] fchunk_units[n_fchunks] fmeta_off[n_fchunks]
 *   fmeta_words[n_fchunks] fmeta[n_fmeta] proc_foff[nnz_l]
 *   [n_pad_b, n_pad_f, dummy_units] pad_boff[n_pad_b] pad_foff[n_pad_f]
 *   chunk_pre_u0[n_chunks] chunk_pre_units[n_chunks]
 *   [frontier_slots, frontier_lag, max_frows] (0, 0, 0 without bit 2) */
/* ------------------------------------------------------------------ */
/* Stage model of the nonlinear SQP workload (a rigid-body quadrotor). */
/* No counterpart in the reference, whose stage functions and their   */
/* derivatives come from CasADi (warpmpc/jax_sqp/casadi_stage.py:     */
/* 66-189; CasADi is absent here).  State x = [p (3), roll/pitch/yaw  */
/* (3), v (3, world), w (3, body rates)], input u = 4 motor thrusts:  */
/*   p' = v;  eta' = W(eta) w;  v' = (sum f)/m R(eta) e3 - g e3;      */
/*   w' = J^-1 (tau - w x J w),  J = diag(jx, jy, jz),                */
/*   tau = (arm (-f1 - f2 + f3 + f4), arm (-f1 + f2 + f3 - f4),       */
/*          yaw_coef (-f1 + f2 - f3 + f4)),                           */
/* discretised with one classical RK4 step of length dt.              */
typedef struct wmpc_quadrotor_model {
  float mass, jx, jy, jz, arm, yaw_coef, gravity;
} wmpc_quadrotor_model;

/* For every stage k < n_stages and instance b: F(x_k, u_k) of the stage
 * variables z[b * z_stride + 16 k + (0..11 | 12..15)] (batch-major z of the
 * SQP, stage blocks of 16) into x_next[(k * batch + b) * 12 + i] and, when
 * jac is not NULL, the dynamics rows' Jacobian entries of g = x_next - F
 * into jac[(k * batch + b) * 126 + e] in wmpc_quadrotor_jac_pattern's order
 * (forward-mode derivatives, float32).  Stream-ordered, launch only. */
int wmpc_quadrotor_rk4(const wmpc_quadrotor_model* model, const float* z, int64_t z_stride, int32_t batch,
                       int32_t n_stages, float dt, float* x_next, float* jac, wmpc_stream_t stream);
/* The entry order of those 126 entries: row_ptr[13] (entries of row r at
 * [row_ptr[r], row_ptr[r + 1])) and cols[126] (0..15 = [x, u] of the stage,
 * 16 + r = x_next,r).  Host only. */
int wmpc_quadrotor_jac_pattern(int32_t* cols, int32_t* row_ptr);

/* Host-only query of the chunk tables the per-call solve (wmpc_solve) uses
 * for its TMA-fed kernel (for CPU-side checks; no counterpart in the
 * reference).  out = [n_chunks, table_words, tables[table_words],
 * desc[8 n_chunks]]; each chunk's table is {columns C, entries E, c0, e0,
 * C column ends relative to e0, E row byte offsets (row * 128)} padded to 4
 * words, its desc {table word offset, table words, e0, c0, E, C, 0, 0}.
 * WMPC_ERR_UNSUPPORTED when a column has more than 64 entries (the solve
 * then runs the one-lane kernel).  With out = NULL only *out_words is set. */
int wmpc_solve_tables_host(const wmpc_pattern_desc* desc, int32_t* out, int64_t out_capacity, int64_t* out_words);
int wmpc_stream_schedule_host(const wmpc_pattern_desc* desc, const float* rho, const float* rhoinv,
                              int32_t n_primal, int32_t units, int32_t cols, int32_t rel, int32_t funits,
                              int32_t offload, int32_t* out, int64_t out_capacity, int64_t* out_words);

/* Profiling (no counterpart in the reference, which times with wall
 * clocks around jax.block_until_ready).  Between begin and end the library
 * records a CUDA event pair on the launching stream around every launch of
 * the dominant kernel (the persistent solve kernel, or the per-call solve
 * kernel of the plain path) and counts every kernel it launches.  end()
 * waits for the recorded events and returns the summed device time. */
int wmpc_profile_begin(void);
int wmpc_profile_end(float* dominant_ms, int32_t* dominant_launches, int64_t* total_launches);
/* Which launches the event pairs bracket: 0 (default) the dominant kernel
 * as above, 1 the factorization kernels (the streaming factorization of
 * the persistent path, the per-call factorization).  No counterpart in the
 * reference. */
int wmpc_profile_select(int32_t channel);
/* The last streaming ADMM launch of this process (no counterpart in the
 * reference): info = {schedule form (0 none yet, 1 plain, 2 frontier),
 * CTAs per SM, grid size, dynamic shared memory bytes}. */
int wmpc_stream_last_launch(int32_t info[4]);
/* Kernels launched by this library since load (or the last profile_begin). */
int64_t wmpc_launch_count(void);

/* ------------------------------------------------------------------ */
/* Adjoint (reverse-mode derivatives of the solution).                 */
/* Replaces CompiledOSQP.adjoint_derivative_compute/get_mat/get_vec    */
/* (solver.py:1046-1192) and the custom_vjp backward rules             */
/* (solver.py:1252-1465).  Instead of the reference's separate adjoint */
/* KKT factorization + refinement, it solves the active-set adjoint    */
/* system  [P A_C^T; A_C 0] [w; mu] = [-dx; t]  (t_r = -tau_r dy_r,    */
/* tau = +1 upper-active / -1 lower-active, equality rows by sign(y))  */
/* as an equality-constrained QP with the forward's ADMM, re-using the */
/* forward's LDL^T factor still held in the workspace.  Outputs follow */
/* the reference's formulas: dq = w, du = -mu (upper rows), dl = -mu   */
/* (lower rows), dP = (w x^T + x w^T)/2 on P's upper pattern,          */
/* dA = y w^T + mu x^T on A's pattern (per instance).                  */
/* ------------------------------------------------------------------ */
typedef struct wmpc_osqp_adjoint_batch {
  int32_t batch;
  const float* p_values; int32_t p_batch;   /* the forward's P/A values   */
  const float* a_values; int32_t a_batch;
  const float* l; const float* u;           /* forward bounds [batch x m] */
  const float* x; const float* z; const float* y; /* forward solution     */
  const float* dx; const float* dy;         /* cotangents; dy may be NULL */
  float* dq; float* dl; float* du;          /* [batch x n], [batch x m]   */
  float* dp; float* da;                     /* [batch x nnz_p], [batch x nnz_a] */
  float* adj_prim_res;                      /* optional [batch]           */
} wmpc_osqp_adjoint_batch;

/* Workspace for a forward solve that keeps its factor for the adjoint
 * (pass the same buffer to wmpc_osqp_solve and wmpc_osqp_adjoint). */
size_t wmpc_osqp_adjoint_workspace_bytes(const wmpc_osqp* osqp, int32_t batch, int32_t mode);
/* options->max_iter: ADMM iterations of the adjoint solve. */
int wmpc_osqp_adjoint(const wmpc_osqp* osqp, const wmpc_osqp_options* options,
                      const wmpc_osqp_adjoint_batch* data, int32_t mode, void* workspace,
                      size_t workspace_bytes, wmpc_stream_t stream);

/* ------------------------------------------------------------------ */
/* Filter line search of the SQP outer loop.                           */
/* ------------------------------------------------------------------ */
/* Reasons (warpmpc/jax_sqp/line_search.py:12-15). */
enum {
  WMPC_LINE_SEARCH_MAX_ITER = 0,            /* nothing accepted: last step of the ladder */
  WMPC_LINE_SEARCH_CONSTRAINT = 1,
  WMPC_LINE_SEARCH_COST = 2,
  WMPC_LINE_SEARCH_COST_OR_CONSTRAINT = 3
};

/* FilterLineSearchSettings (line_search.py:18-29), in float32; the step
 * ladder itself (make_step_lengths, line_search.py:45-59) is host data. */
typedef struct wmpc_line_search_settings {
  float g_max;                  /* line_search_g_max          (1e-1) */
  float g_min;                  /* line_search_g_min          (1e-3) */
  float gamma_c;                /* line_search_gamma_c        (1e-3) */
  float armijo_factor;          /* line_search_armijo_factor  (1e-4) */
  float constraint_scale;       /* line_search_constraint_scale (0.1) */
  int32_t cost_accept_uses_trial_cost; /* 1 (reference default) or 0 */
} wmpc_line_search_settings;

/* constraint_violation (line_search.py:62-69): out[b] = scale *
 * sqrt(sum_r max(l - g, 0)^2 + sum_r min(u - g, 0)^2) over batch-major
 * [batch x m] rows. */
int wmpc_constraint_violation(const float* lower, const float* g, const float* upper, int32_t batch,
                              int32_t m, float scale, float* out, wmpc_stream_t stream);

/* filter_line_search_from_evaluations (line_search.py:72-169).  Candidate
 * arrays are [n_candidates x batch] (row k = step k of the ladder); the
 * selected index is the first accepted candidate, else n_steps - 1, and the
 * candidate/step gathers clamp it into range.  cost, violation, reason,
 * accepted and candidate_acceptance ([n_candidates x batch], 0/1) may be
 * NULL.  Replaces the jnp computation; bit-exact with a float32 restatement. */
int wmpc_filter_line_search(const wmpc_line_search_settings* settings, const float* step_lengths,
                            int32_t n_steps, const float* baseline_cost, const float* baseline_violation,
                            const float* armijo_metric, const float* candidate_costs,
                            const float* candidate_violations, int32_t n_candidates, int32_t batch,
                            float* step_length, float* cost, float* violation, int32_t* reason,
                            uint8_t* accepted, uint8_t* candidate_acceptance, wmpc_stream_t stream);

/* The line-search SQP step after its QP solve (sparse_mpc.py:1013-1052), one
 * launch: the baseline violation of (constraint_l, g, constraint_u), the
 * Armijo metric q . direction, the filter selection over the candidates'
 * evaluations (costs and violations of z + step_k direction, computed by the
 * caller's NLP), z_next = z + step direction and is_finite.  Batch-major
 * [batch x n] / [batch x m]; outputs other than z_next and step_length may
 * be NULL. */
typedef struct wmpc_sqp_step_batch {
  int32_t batch, n, m, n_steps, n_candidates;
  const float* step_lengths;                    /* [n_steps] */
  const float* z; const float* direction;       /* [batch x n] */
  const float* q;                               /* linearization's q [batch x n] */
  const float* constraint_l; const float* g; const float* constraint_u; /* [batch x m] */
  const float* baseline_cost;                   /* [batch] */
  const float* candidate_costs;                 /* [n_candidates x batch] */
  const float* candidate_violations;            /* [n_candidates x batch] */
  float* z_next;                                /* [batch x n] */
  float* step_length; float* cost; float* violation; float* baseline_violation; /* [batch] */
  int32_t* reason; uint8_t* accepted; uint8_t* is_finite; /* [batch] */
  uint8_t* candidate_acceptance;                /* [n_candidates x batch] */
} wmpc_sqp_step_batch;
int wmpc_sqp_line_search_step(const wmpc_line_search_settings* settings, const wmpc_sqp_step_batch* data,
                              wmpc_stream_t stream);

/* ------------------------------------------------------------------ */
/* Reference-style adjoint (parity mode) helper.                       */
/* ------------------------------------------------------------------ */
/* y = S x - r per instance (r may be NULL: y = S x), S symmetric with one
 * pattern: `values` holds its upper triangle symbolic-major
 * ([nnz x batch], leading dimension values_ld); the device table
 * row_ptr[n+1] / ent_pos / ent_col lists, per row i, the (value position,
 * column) terms of the full symmetric pattern.  x, r, y are [n x batch];
 * y must not alias x.  Replaces _adjoint_matvec (warpmpc/jax_osqp/
 * solver.py:1035-1044) in the refinement loop of the reference's adjoint
 * solve (1133-1141), whose factor and solves run on wmpc_factor /
 * wmpc_solve. */
int wmpc_sym_matvec(const int32_t* row_ptr, const int32_t* ent_pos, const int32_t* ent_col, int32_t n,
                    const float* values, int64_t values_ld, const float* x, const float* r, float* y,
                    int32_t batch, wmpc_stream_t stream);

/* ------------------------------------------------------------------ */
/* Sparse MPC QP assembly (SQP linearization).                         */
/* ------------------------------------------------------------------ */
typedef struct wmpc_sqp_assemble_dims {
  int32_t batch, n, nnz_p, nnz_a, m, n_stages, width;
} wmpc_sqp_assemble_dims;

/* The scatter half of _linearize_jit (warpmpc/jax_sqp/sparse_mpc.py:
 * 855-901): values [batch x width] hold each instance's packed stage
 * values (per stage: cost, g, lower, upper, grad, hess, jac).  Device
 * tables: add_ptr[n + nnz_p + nnz_a + 1] / add_src list, for every entry of
 * [q | P values | A values], the value columns added into it, in stage
 * order (summed from zero in that order); row_src[2 m] the g column of
 * each constraint row, then its stage's constraint_dim (lower and upper sit
 * that far and twice that far after g); cost_src[n_stages] the cost
 * columns.  Outputs batch-major: q [batch x n], p_values, a_values, l =
 * lower - g, u = upper - g, g, constraint_l (lower), constraint_u (upper)
 * [batch x m], cost [batch]. */
int wmpc_sqp_assemble(const wmpc_sqp_assemble_dims* dims, const int32_t* add_ptr, const int32_t* add_src,
                      const int32_t* row_src, const int32_t* cost_src, const float* values, float* q,
                      float* p_values, float* a_values, float* l, float* u, float* cost, float* g,
                      float* constraint_l, float* constraint_u, wmpc_stream_t stream);

const char* wmpc_last_error_string(void);
/* Library version string, e.g. "0.1.0 sm_100a". */
const char* wmpc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WARPMPC_B200_H */
