/*
 * mguso_cuda.h -- C ABI of the B200-native (sm_100a) mguso implicit-step library.
 *
 * This is the drop-in boundary for the reference engine's implicit IPC step
 * (SeedeXR/nguo-3d, core-engine). Every entry point takes plain pointers and sizes,
 * returns an int status (MGUSO_OK = 0) and records a message readable through
 * mguso_last_error(). Handles are opaque; one handle is used by one thread at a time
 * (the reference's LinearSolver is not Sync either: linsolve.rs:415-442).
 *
 * Pointer conventions: arguments documented as "host" are caller-owned host memory;
 * arguments documented as "device" are device pointers on the context's GPU, used on
 * the given CUDA stream (NULL = the legacy default stream).
 */
#ifndef MGUSO_CUDA_H
#define MGUSO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define MGUSO_OK 0
#define MGUSO_ERR_INVALID_ARG 1   /* bad pointer, size or parameter */
#define MGUSO_ERR_OOM 2           /* device allocation failed */
#define MGUSO_ERR_NONFINITE 3     /* a step produced NaN/Inf and was rejected */
#define MGUSO_ERR_PCG_CAP 4       /* PCG hit max_iter before reaching tol */
#define MGUSO_ERR_CCD_CAP 5       /* a CCD root solve hit its iteration cap */
#define MGUSO_ERR_PAIR_OVERFLOW 6 /* candidate-pair buffer too small (count still reported) */
#define MGUSO_ERR_BVH_STACK 7     /* LBVH traversal stack overflow */
#define MGUSO_ERR_CUDA 8          /* a CUDA runtime call failed */
#define MGUSO_ERR_TIMEOUT 9       /* a bounded device wait gave up */
#define MGUSO_ERR_UNSUPPORTED 10  /* configuration not supported */

/* Preconditioners (linsolve.rs:67-76). */
#define MGUSO_PRECOND_BLOCK_JACOBI 1
#define MGUSO_PRECOND_SCHWARZ 2

/* Arithmetic of the PCG reductions: FP32 everywhere, or FP64 dots/norms (MIXED). */
#define MGUSO_PRECISION_FP32 0
#define MGUSO_PRECISION_MIXED 1

typedef struct mguso_ctx mguso_ctx;
typedef struct mguso_bsr mguso_bsr;
typedef struct mguso_schwarz mguso_schwarz;
typedef struct mguso_linear_solver mguso_linear_solver;

/* Library version (major*10000 + minor*100 + patch). */
int mguso_version(void);

/* Copies the calling thread's last error message (NUL-terminated, truncated to len).
 * Returns the full message length. */
size_t mguso_last_error(char* buf, size_t len);

/* GPU context: selects `device` and owns a stream. The reference's GpuContext::new()
 * (engine-gpu/src/lib.rs:91-126). */
int mguso_ctx_create(int device, mguso_ctx** out);
/* Every object created on a context (solvers, operators, scenes, batches, BVHs, adjoints)
 * uses its stream and must be destroyed before the context is. */
int mguso_ctx_destroy(mguso_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t). */
void* mguso_ctx_stream(mguso_ctx* ctx);

/* Scalar CSR as the reference builds it (CsrMatrix, engine-core/src/csr.rs:9-14): square
 * n x n, n = 3 * vertices, columns sorted within each row. All pointers host. */
typedef struct {
  uint32_t n;
  const uint32_t* row_ptr; /* n + 1 */
  const uint32_t* col_idx; /* row_ptr[n] */
  const float* values;     /* row_ptr[n] */
} mguso_csr;

typedef struct {
  uint32_t iters;   /* PCG iterations performed */
  double residual;  /* final relative residual ||r|| / ||b|| */
  int status;       /* MGUSO_OK, or MGUSO_ERR_PCG_CAP when max_iter was reached */
} mguso_lin_stats;

/* ---- LinearSolver (replaces engine_core::LinearSolver, linsolve.rs:21-28) ----------- */
/* A stateful solver like SchwarzCpu (linsolve.rs:463-520): caches the block pattern,
 * BSR layout and Schwarz domains while the sparsity is unchanged. `domain` is the
 * Schwarz domain size in vertices (ignored for block Jacobi). */
int mguso_linear_solver_create(mguso_ctx* ctx, int precond, uint32_t domain, int precision,
                               mguso_linear_solver** out);
/* The two-level variant, SchwarzMlCpu::new(domain, weight) (linsolve.rs:779-836): z =
 * S0 r + weight * C1^T S1 (C1 r), with the Galerkin coarse operator rebuilt from the matrix
 * values at every solve (the reference's CLI default is domain 16, weight 0.7). */
int mguso_linear_solver_create_ml(mguso_ctx* ctx, uint32_t domain, float weight, int precision,
                                  mguso_linear_solver** out);
int mguso_linear_solver_destroy(mguso_linear_solver* s);
/* solve(a, b, tol, max_iter) -> x  (LinearSolver::solve). a, b, x host; x has a->n
 * entries. Stats as LinearSolver::last_stats. Reaching max_iter is reported in
 * stats->status; the return value is still MGUSO_OK and x holds the last iterate, as in
 * the reference, which returns the best x without failing. */
int mguso_linear_solve(mguso_linear_solver* s, const mguso_csr* a, const float* b, float tol,
                       uint32_t max_iter, float* x, mguso_lin_stats* stats);

/* ---- Device-resident 3x3 BSR operator ----------------------------------------------- */
/* Builds a device BSR from a host scalar CSR whose 3x3 block structure is implied by the
 * vertex grouping (every vertex pair contributes 9 entries, implicit.rs:2394-3103).
 * Missing entries inside a present block are stored as 0. */
int mguso_bsr_create_from_csr(mguso_ctx* ctx, const mguso_csr* a, mguso_bsr** out);
/* Builds a device BSR directly from host block arrays: nb block rows, row_ptr (nb+1),
 * col (nnzb) sorted per row, val (9*nnzb, row-major 3x3 per block). */
int mguso_bsr_create(mguso_ctx* ctx, uint32_t nb, const uint32_t* row_ptr, const uint32_t* col,
                     const float* val, mguso_bsr** out);
int mguso_bsr_destroy(mguso_bsr* a);
int mguso_bsr_info(const mguso_bsr* a, uint32_t* nb, uint32_t* nnzb);
/* y = A x with x, y device (3*nb floats each), on `stream`. */
int mguso_bsr_spmv(mguso_bsr* a, const float* x, float* y, void* stream);
/* y = A x with x, y host: copies in, multiplies, copies out (synchronous). */
int mguso_bsr_spmv_host(mguso_bsr* a, const float* x, float* y);
/* Selects the SpMV kernel variant: 0 = auto (autotuned), 1 = TMA-staged tiles,
 * 2 = direct thread-per-row, 3 = sliced ELL (32-row slices, coalesced 128-byte loads;
 * builds the sliced copy on first use). Returns the variant in use through *active. */
int mguso_bsr_set_kernel(mguso_bsr* a, int variant, int* active);
/* Runs the SpMV autotuner on this matrix (times every variant and tile shape with CUDA
 * events) and keeps the fastest. *best_us gets its time per apply. */
int mguso_bsr_autotune(mguso_bsr* a, float* best_us);
/* The variant in use (1 TMA, 2 direct, 3 sliced ELL; 0 before any choice) and, for TMA,
 * its tile shape (block rows per tile, pipeline stages; 0 otherwise). */
int mguso_bsr_kernel(const mguso_bsr* a, int* variant, int* tile_rows, int* stages);

/* ---- One-level additive Schwarz preconditioner (linsolve.rs:126-258) --------------- */
/* Domains are greedy BFS aggregates of <= `domain` vertices over the block graph of `a`
 * (linsolve.rs:152-173); vertices without off-diagonal blocks are packed `domain` at a
 * time. Each domain's dense block (with the reference's diagonal floor) is
 * Cholesky-factored in FP64 and W = L^-1 stored in FP32 (32 x 32 tiles of its lower
 * block-triangle); the apply is z = W^T (W r) per domain, symmetric positive definite for
 * any rounding of W. factor_bytes reports the stored tile bytes. */
int mguso_schwarz_create(mguso_bsr* a, uint32_t domain, mguso_schwarz** out);
int mguso_schwarz_destroy(mguso_schwarz* s);
int mguso_schwarz_info(const mguso_schwarz* s, uint32_t* ndomains, uint64_t* factor_bytes);
/* Re-factors every domain from the current values of `a` (device, on `stream`). */
int mguso_schwarz_factor(mguso_schwarz* s, void* stream);
/* z = M^-1 r with r, z device (3*nb floats), on `stream`. */
int mguso_schwarz_apply(mguso_schwarz* s, const float* r, float* z, void* stream);
/* Domain id of every vertex (host, nb entries). */
int mguso_schwarz_domains(const mguso_schwarz* s, uint32_t* dom_of_vertex);
/* Two-level Galerkin additive Schwarz (MultilevelSchwarz, linsolve.rs:534-666):
 * z = S0 r + weight * C1^T S1 (C1 r). S0 is the one-level apply above (here every vertex
 * without off-diagonal blocks is a domain of its own, as in the reference); C1 sums a
 * vertex's residual into its domain (one coarse node of three dofs per domain); S1 is a
 * one-level Schwarz over the Galerkin operator A1 = C1 A C1^T whose domains are BFS groups of
 * <= `domain` coarse nodes. mguso_schwarz_factor factors both levels (the coarse blocks are
 * summed in FP32 in the order of the fine values, as coarse_matrix, linsolve.rs:618-630). */
int mguso_schwarz_create_ml(mguso_bsr* a, uint32_t domain, float weight, mguso_schwarz** out);
/* Coarse domain of every coarse node (= level-0 domain; host, one entry per domain). */
int mguso_schwarz_coarse_domains(const mguso_schwarz* s, uint32_t* coarse_dom_of_domain);

/* ---- LBVH broad phase (engine-gpu/src/{morton,radix,karras,bvh_aabb,bvh_traverse}.rs) */
/* Triangle BVH: 30-bit (u32) or 63-bit (u64) Morton codes of the centroids normalised by
 * the centroid box (morton.rs:21-63), a stable onesweep radix sort of (code, triangle),
 * the Karras tree (karras.rs:24-88) and exact min/max node boxes (bvh_aabb.rs:28-56). */
typedef struct mguso_lbvh mguso_lbvh;
int mguso_lbvh_create(mguso_ctx* ctx, mguso_lbvh** out);
int mguso_lbvh_destroy(mguso_lbvh* b);
/* positions f32[3*nv], tris u32[3*nt] device; key_bits 30 or 63. */
int mguso_lbvh_build(mguso_lbvh* b, const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt,
                     int key_bits, void* stream);
/* Emits (query, triangle) for every leaf box overlapping [p - dhat, p + dhat]
 * (bvh_traverse.wgsl:64-92): points f32[3*np], pairs u32[2*cap], *count (u64) device.
 * *count receives the total even when it exceeds cap (then status = PAIR_OVERFLOW).
 * Queries are visited in Morton order so a warp walks neighbouring points together. */
int mguso_lbvh_query_points(mguso_lbvh* b, const float* points, uint32_t np, float dhat, uint32_t* pairs,
                            uint64_t cap, uint64_t* count, void* stream);
/* Host copies of the last build: keys (zero-extended to u64), perm, left/right (nt-1),
 * node boxes f32[6*(nt-1)] as [lo.xyz, hi.xyz]. Any pointer may be NULL. */
int mguso_lbvh_download(mguso_lbvh* b, uint64_t* keys, uint32_t* perm, uint32_t* left, uint32_t* right,
                        float* node_boxes);
/* Device status of the last build/query: MGUSO_OK, MGUSO_ERR_PAIR_OVERFLOW,
 * MGUSO_ERR_BVH_STACK or MGUSO_ERR_TIMEOUT (synchronises the context stream). */
int mguso_lbvh_status(mguso_lbvh* b);
/* enable != 0 records per-stage events; ms6 receives the last build+query's stage times:
 * morton, sort, karras, refit, query preparation, traversal (ms). */
int mguso_lbvh_stage_times(mguso_lbvh* b, int enable, float* ms6);
/* Host-buffer convenience over build + point query (the operator entry point a binding
 * calls): out_keys (u64[nt]), out_perm (u32[nt]) and out_pairs (u32[2*cap]) may be NULL. */
int mguso_lbvh_build_query(mguso_ctx* ctx, const float* positions, uint32_t nv, const uint32_t* tris,
                           uint32_t nt, int key_bits, float dhat, uint64_t* out_keys, uint32_t* out_perm,
                           uint32_t* out_pairs, uint64_t cap, uint64_t* count);
/* Stable onesweep LSD radix sort of (key, u32 payload) pairs in place (device pointers):
 * u32 keys when key_bits <= 32, u64 keys otherwise. Replaces GpuRadixSort::sort_pairs
 * (radix.rs:112-352), which is limited to 65 536 keys. */
int mguso_radix_sort_pairs(mguso_ctx* ctx, void* keys, uint32_t* vals, uint32_t n, int key_bits, void* stream);
/* Waits for the device, then reports whether the last mguso_radix_sort_pairs of this context
 * gave up a bounded look-back wait (MGUSO_ERR_TIMEOUT; its output is then not sorted). */
int mguso_radix_sort_status(mguso_ctx* ctx);
/* Allocation-free variant of mguso_radix_sort_pairs, with no counterpart in the reference.
 * For callers that may not allocate device memory once they are running (a host engine
 * that gives all of the GPU's memory to its own pool at start-up, or a per-frame path that
 * cannot afford cudaMalloc's device-wide synchronisation): it allocates nothing and needs
 * no context. Its temporaries live in one fixed 3.2 MiB device array inside this library
 * (on every device that loads it, until the process exits), which limits n to 262 144
 * pairs; larger n returns MGUSO_ERR_INVALID_ARG. Sorts the same (key, payload) pairs in
 * place on the current device, stably, with the same result as mguso_radix_sort_pairs, and
 * returns when the sort has finished on `stream`. The first call on each device does a
 * one-time set-up: it looks up the array's device address and keeps it for the life of the
 * process, so make that first call before any stream capture begins. After cudaDeviceReset
 * on a device the kept address is stale, so a process that resets a device must not call
 * this function on it again. All calls share the one array, so calls that overlap on the
 * GPU (other streams, other host threads) race and must be serialised by the caller. */
int mguso_radix_sort_pairs_noalloc(void* keys, uint32_t* vals, uint32_t n, int key_bits, void* stream);

/* ---- Implicit step: scene build -> step -> readback --------------------------------- */
/* Solver knobs, named and defaulted as ImplicitParams (implicit.rs:30-229). Fields that
 * the reference does not have: newton_tol (Newton stops once the largest per-vertex step
 * actually taken is below it, 0 = off), precond/schwarz_domain (the LinearSolver choice)
 * and precision (MGUSO_PRECISION_FP32, or MIXED = FP64 PCG dots and norms, FP64 contact
 * distances/barriers and FP64 CCD root solves). barrier_kind: 0 log, 1 cubic. */
typedef struct {
  float dt;
  float gravity[3];
  uint32_t newton_iters;
  float stiffness;      /* stretch-spring k on the unique mesh edges */
  float bend_stiffness; /* hinge k_b (hinge weight w = 1) */
  float max_dx;         /* search-direction cap (INFINITY = off) */
  float target_toi;
  uint32_t min_newton_steps;
  uint32_t ccd_max_iter;
  float eiganalysis_eps;
  float contact_dhat;
  float contact_kappa;
  float contact_dynamic;
  float shell_mu;
  float shell_lambda;
  float friction;
  float friction_eps;
  int barrier_kind;
  int contact_rayleigh;
  int self_collision;
  float cg_tol;
  uint32_t cg_max_iter;
  float floor_y; /* -INFINITY = off */
  float newton_tol;
  int precond;
  uint32_t schwarz_domain;
  int precision;
  int pcg_mode;            /* 0: two fused kernels per iteration (rows, domains) at full
                                 occupancy, replayed as CUDA graphs (default);
                              1: one launch per PCG kernel, replayed as CUDA graphs (single
                                 scenes only);
                              2: one cooperative persistent launch per linear solve */
  int factor_storage;      /* Schwarz factor tiles: 0 = by precision (FP32 tiles with
                              MGUSO_PRECISION_FP32, FP16 tiles scaled per domain with MIXED),
                              1 = FP32 tiles, 2 = FP16 tiles */
  uint32_t schwarz_levels; /* 1 (or 0): one-level Schwarz (SchwarzCpu, linsolve.rs:463-520);
                              2: two-level Galerkin Schwarz (SchwarzMlCpu, linsolve.rs:534-836) */
  int pcg_variant;         /* kernels of the fused PCG (pcg_mode 0): 0 = chosen by the autotuner
                              at the scene's first solve (cached per system size); v in 1..24
                              fixes the rows kernel (v - 1) / 6 (0, 1, 2: 2, 1 or 4 lanes per
                              block row over the BSR; 3: one lane per row over a sliced-ELL copy)
                              and the Schwarz domain kernel (v - 1) % 6 (0: one warp per domain,
                              4 per CTA; 1, 2, 3: three warps per domain, 1, 2 or 4 domains per
                              CTA; 4, 5: FP16 tiles on the tensor cores, one warp per domain, 4
                              or 8 per CTA, else as 0) */
  float membrane_warp;     /* Baraff-Witkin membrane stiffnesses (ImplicitParams::membrane_warp /
                              _weft / _shear, implicit.rs:39-43): 0 = off. The membrane covers
                              every triangle of tris, rest shape from the initial positions */
  float membrane_weft;
  float membrane_shear;
  float constraint_tol;    /* pin gap floor as a fraction of the pin's ghat (0 = 1e-2, the
                              reference's default ImplicitParams::constraint_tol) */
  float schwarz_weight;    /* coarse-correction weight w of the two-level form
                              z = S0 r + w C1^T S1 (C1 r) (the CLI default 0.7, main.rs:761-763) */
  float strain_limit_ratio; /* one-sided edge strain limit (ImplicitParams::strain_limit_ratio,
                               _k, _ratio_weft, implicit.rs:160-170; strain_limit.rs:24-63): on
                               every stretch edge a spring of rest length ratio * rest and
                               stiffness strain_limit_k, active only while the edge is longer;
                               0 = off */
  float strain_limit_k;
  float strain_limit_ratio_weft; /* > 0 with per-vertex uvs: edges more V- than U-aligned in UV
                                    space use this ratio instead (edge_strain_ratio,
                                    implicit.rs:798-817) */
} mguso_params;

/* One scene (Scene::build_implicit + the set_* calls of implicit.rs). All pointers host;
 * they are copied, the caller keeps ownership. */
typedef struct {
  uint32_t nv;
  const float* positions;   /* f32[3*nv] */
  const float* velocities;  /* f32[3*nv] or NULL (zero) */
  const float* inv_mass;    /* f32[nv]; 0 = pinned / static */
  uint32_t nt;
  const uint32_t* tris;     /* u32[3*nt]: every triangle (cloth and bodies): hinges, springs and collision */
  const uint8_t* static_mask; /* u8[nv] static mesh collider vertices, or NULL (set_static_collider_verts) */
  uint32_t nshell;
  const uint32_t* shell_faces; /* u32[3*nshell] StVK shell faces (set_shell_faces) */
  uint32_t nstitch;
  const uint32_t* stitch_idx;  /* u32[6*nstitch] (Stitch::index) */
  const float* stitch_w;       /* f32[6*nstitch] (Stitch::weight) */
  const float* stitch_kl;      /* f32[3*nstitch]: stiffness, l0, l_cap */
  uint32_t ncollider;
  const float* colliders;      /* f32[8*ncollider]: kind (0 half-space, 1 sphere), point/center xyz,
                                  normal xyz, radius (Collider, contact.rs:21-31) */
  mguso_params params;
  /* Optional per-shell-face overrides (NULL: rest shape from the initial positions and the
   * scene's (shell_mu, shell_lambda), as Scene::build_implicit does). shell_rest: 5 floats per
   * face, the inverse rest shape (column-major 2x2) and the rest area; shell_stiff: a factor
   * on (shell_mu, shell_lambda) per face. Used for sewing-pattern rest shapes and for the
   * parameters of the adjoint. */
  const float* shell_rest;
  const float* shell_stiff;
  /* Optional per-vertex pattern coordinates (SimState::uvs), f32[2*nv] or NULL: they choose
   * each edge's strain-limit ratio (strain_limit_ratio_weft). */
  const float* uvs;
  /* Optional stretch edges (SimState::edges), u32[2*nstretch]: when nstretch > 0 the stretch
   * springs and the edge strain limit act on these edges, rest lengths from the initial
   * positions, instead of on the unique edges of tris. Collision edges stay those of tris. */
  uint32_t nstretch;
  const uint32_t* stretch_edges;
} mguso_scene_desc;

typedef struct {
  uint32_t newton_iters;
  uint32_t max_cg_iters;
  uint32_t num_contacts;   /* free vertices within dhat of an analytic collider */
  uint32_t stencils;       /* largest active self-contact stencil count over the Newton iterations */
  uint32_t ccd_cap_hits;   /* CCD root solves that hit ccd_max_iter */
  double max_reresid;
  double t_min;            /* smallest CCD step fraction of the step */
  int penetration_free;
  int all_finite;
  int status;              /* MGUSO_OK, MGUSO_ERR_NONFINITE (step rejected), ... */
} mguso_step_stats;

typedef struct mguso_scene mguso_scene;
/* Checks a description without building anything (host only: needs no device or context):
 * index ranges, the stitch rules of ImplicitSolver::set_stitches (implicit.rs:939-966: every
 * index in range, stiffness finite and >= 0, l0 finite and > 0, l_cap finite and >= l0, each
 * side's weights summing to 1 within 1e-3) and the parameters. MGUSO_OK, or
 * MGUSO_ERR_INVALID_ARG with the reason in mguso_last_error, as mguso_scene_create would
 * return for it; the reference's setters return the same rules as Result<(), String>. */
int mguso_scene_validate(const mguso_scene_desc* desc);
int mguso_scene_create(mguso_ctx* ctx, const mguso_scene_desc* desc, mguso_scene** out);
int mguso_scene_destroy(mguso_scene* s);
/* Advances nsteps implicit steps (ImplicitSolver::step, implicit.rs:1951-2191). stats has
 * nsteps * (instances, 1 for a single scene) entries, step-major, or is NULL. A non-finite step is rejected exactly as the reference does
 * (positions kept, velocities zeroed) and reported as MGUSO_ERR_NONFINITE in its stats. */
int mguso_step(mguso_scene* s, int nsteps, mguso_step_stats* stats);

/* A batch of independent drapes (for example one pattern graded into sizes) as one scene:
 * the n <= 8 descriptions are concatenated, so positions and velocities are read and
 * written as one array with instance k at vertices [offsets[k], offsets[k+1]). Every
 * instance runs its own Newton loop (its own termination, CCD step fraction and PCG
 * convergence); the instances still iterating share each launch, and each PCG iteration's
 * kernels cover all of them (pcg_mode 0 or 2). All descriptions must share params and
 * analytic colliders.
 * mguso_step then writes nsteps * n stats, step-major. No counterpart in the reference,
 * which steps one scene at a time. */
int mguso_batch_create(mguso_ctx* ctx, const mguso_scene_desc* descs, uint32_t n, mguso_scene** out);
/* Number of instances and their vertex offsets (u32[n + 1]; may be NULL). */
int mguso_scene_instances(mguso_scene* s, uint32_t* n, uint32_t* vert_offsets);

/* ---- Adjoint of an N-step drape ------------------------------------------------------- */
/* Gradients of a loss on the final positions with respect to sewing-pattern parameters, as a
 * forward/backward pair mirroring torch.autograd.Function (forward(theta) -> x_N,
 * backward(dL/dx_N) -> dL/dtheta). No counterpart in the reference, which has no
 * differentiation. theta has 3 npanel + nseam entries:
 *   [stiff_0 .. stiff_{P-1}, warp_0, weft_0, .., warp_{P-1}, weft_{P-1}, seam_0 .. seam_{S-1}]
 * stiff_p multiplies (shell_mu, shell_lambda) of panel p's shell faces; a face rests at its
 * pattern triangle (shell_uv) scaled by weft_p along u and warp_p along v; seam_q multiplies
 * the stiffness of seam q's stitches. The backward pass solves, per step and in reverse,
 * H w = a_x + a_v / h with H the exact Hessian of the step at its converged positions
 * (symmetric, possibly indefinite: no eigenvalue clamps, with the second-derivative terms of
 * hinges and barriers) by MINRES to a relative residual of 1e-10 (FP64 products with the
 * stored FP32 blocks), preconditioned by the
 * step's own preconditioner factored from its projected matrix, recomputing the states
 * between checkpoints taken every `checkpoint_every` steps. A contact stiffness's dependence
 * on the gap enters H, its dependence on the elastic blocks does not; friction must be 0.
 * MGUSO_ERR_PCG_CAP when MINRES reaches max(cg_max_iter, 4000) iterations. */
typedef struct {
  uint32_t npanel, nseam;
  const float* shell_uv;       /* 6 per shell face: u0 v0 u1 v1 u2 v2 (pattern coordinates) */
  const uint8_t* shell_panel;  /* per shell face */
  const uint8_t* stitch_seam;  /* per stitch */
} mguso_adjoint_spec;
typedef struct mguso_adjoint mguso_adjoint;
int mguso_adjoint_create(mguso_ctx* ctx, const mguso_scene_desc* desc, const mguso_adjoint_spec* spec,
                         mguso_adjoint** out);
int mguso_adjoint_destroy(mguso_adjoint* a);
/* Runs nsteps steps at theta from the description's initial state; x_out f32[3 nv] gets the
 * final positions, stats (optional) nsteps entries. */
int mguso_adjoint_forward(mguso_adjoint* a, const double* theta, uint32_t nsteps, uint32_t checkpoint_every,
                          float* x_out, mguso_step_stats* stats);
/* dl_dx f32[3 nv] (dL/dx_N) -> dl_dtheta f64[3 npanel + nseam], for the last forward. */
int mguso_adjoint_backward(mguso_adjoint* a, const float* dl_dx, double* dl_dtheta);
/* The last forward pass's states x_n and v_n, n = 0..nsteps, recomputed from its checkpoints
 * exactly as the backward pass recomputes them: x_all and v_all host, (nsteps + 1) * 3 nv
 * floats each (state n at offset 3 nv n). */
int mguso_adjoint_states(mguso_adjoint* a, float* x_all, float* v_all);
int mguso_read_positions(mguso_scene* s, float* out);   /* f32[3*nv] host */
int mguso_write_positions(mguso_scene* s, const float* in);
int mguso_read_velocities(mguso_scene* s, float* out);
int mguso_write_velocities(mguso_scene* s, const float* in);
/* Move the scene's static mesh collider (its vertices of static_mask) to x (f32[3 nv]; other
 * rows are ignored) between steps: those vertices take x and the velocity of that move over
 * one step, and the collider's pseudonormals are recomputed. MGUSO_ERR_INVALID_ARG, with
 * nothing written, when the scene has no static collider or a collider row of x is not
 * finite. The next step's CCD sees the collider already at x (the body teleports, as in the
 * reference). Counterpart: ImplicitSolver::set_kinematic_collider_positions
 * (core-engine/crates/engine-core/src/implicit.rs:1368-1398). */
int mguso_set_kinematic_collider_positions(mguso_scene* s, const float* x);
/* set_pins (implicit.rs:826-838): n pins (the reference's FixPair, implicit.rs:230-262), each
 * confining vertex index[i] to a ball of radius ghat[i] around target[3 i..] with the dynamic
 * stiffness (H w).w / |w|^2 + m / gap^2 (w = x - target, H the vertex's elastic diagonal
 * block, gap = max(ghat - |w|, constraint_tol ghat)); a kinematic pin's stiffness is scaled
 * by stiffness[i] and takes no part in the CCD, a static pin's ball limits the step fraction
 * (implicit.rs:1755-1789). kinematic and stiffness may be NULL (all static, 1). All or
 * nothing: an index out of range or a ghat <= 0 returns MGUSO_ERR_INVALID_ARG and keeps the
 * previous pins; n = 0 clears them. All pointers host. */
int mguso_set_pins(mguso_scene* s, uint32_t n, const uint32_t* index, const float* target, const float* ghat,
                   const uint8_t* kinematic, const float* stiffness);
/* set_pulls (implicit.rs:852-864): n pulls (PullPair, implicit.rs:264-282), each adding
 * weight[i] |x - target|^2 / 2 on vertex index[i]. All or nothing: an index out of range or
 * a weight <= 0 returns MGUSO_ERR_INVALID_ARG and keeps the previous pulls; n = 0 clears
 * them. All pointers host. */
int mguso_set_pulls(mguso_scene* s, uint32_t n, const uint32_t* index, const float* target, const float* weight);
/* set_strain_limit_faces (implicit.rs:1088-1121): the per-face strain-limit barrier
 * (shell_model.rs:438-640) on n faces (u32[3 n]), each with its allowed principal-stretch
 * excess limits[i] (0.05 = 5 %) and its mass masses[i]; the rest shape comes from the
 * current positions. Faces with a limit or mass <= 0, and degenerate faces, are skipped;
 * *kept (may be NULL) gets the number kept. Each kept face adds the barrier on
 * max(sigma - 1) at the dynamic stiffness max(w.(H w), 0) + mass / d^2 (w the face's
 * positions about their centroid, H the elastic blocks gathered so far, d the headroom),
 * and limits the step fraction by bisection (implicit.rs:1709-1753). All or nothing:
 * MGUSO_ERR_INVALID_ARG for an index out of range, a face across two instances of a batch
 * or a non-finite limit or mass; MGUSO_ERR_UNSUPPORTED when a face has two vertices, one of
 * them free, that share no element (the barrier's block would lie outside the scene's
 * fixed Hessian pattern). n = 0 clears them. All pointers host. */
int mguso_set_strain_limit_faces(mguso_scene* s, uint32_t n, const uint32_t* faces, const float* limits,
                                 const float* masses, uint32_t* kept);
/* Element counts: hinges, shells, unique edges, static collider triangles,
 * system blocks (free-free pattern), pinned-pattern blocks. */
int mguso_scene_info(mguso_scene* s, uint32_t* out6);
/* Times `reps` applications of the scene's current system operator y = (Ps + C) x on the
 * context stream with CUDA events (the PCG's SpMV at the last Newton iterate): *us gets the
 * mean time per apply, *bytes its algorithmic bytes (blocks, columns, row pointers, x, y). */
int mguso_scene_spmv_time(mguso_scene* s, int reps, float* us, double* bytes);

/* Mean device time in microseconds of the step's linear-solver kernels at the last
 * assembled system, each timed alone over `reps` launches with CUDA events on the scene's
 * stream: us4 = {system SpMV, preconditioner apply, preconditioner factorisation, PCG
 * vector update}; bytes4 = their algorithmic bytes per launch (each stored block or factor
 * entry and each vector read or written once). Clobbers the PCG scratch (not the state). */
int mguso_scene_profile(mguso_scene* s, int reps, float* us4, double* bytes4);

/* Mean device time in microseconds of the two fused PCG kernels (pcg_mode 0 and batches)
 * inside a solve of the last assembled system: `iters` iterations of every instance at
 * tolerance 0, each launch bracketed by its own CUDA events on the scene's stream, so the
 * kernels see the cache state of a real solve. us2 = {rows kernel (direction update, system
 * SpMV, p.Ap), domain kernel (x/r update, preconditioner apply, r.r and r.z)}; bytes2 =
 * their algorithmic bytes per launch. Clobbers the PCG scratch (not the state). */
int mguso_scene_profile_pcg(mguso_scene* s, int iters, float* us2, double* bytes2);
/* The fused PCG kernels in use, as the autotuner (or pcg_variant) chose them: out2 = {rows
 * kernel: 0 two lanes per block row, 1 one, 2 four, 3 sliced ELL; domain kernel: 0 one warp per domain and
 * four domains per CTA, 1/2/3 three warps per domain and 1/2/4 domains per CTA}; -1 before
 * the scene's first solve. */
int mguso_scene_pcg_kernels(mguso_scene* s, int* out2);

/* The self-intersection scan behind mguso_step_stats.penetration_free
 * (ImplicitSolver::has_self_intersection, implicit.rs:618-650): at positions x (host
 * f32[3 nv]; the scene's positions are left at x), counts[k] gets instance k's number of
 * (mesh edge, collision triangle) pairs that share no vertex, have a movable vertex, and
 * where the edge crosses the triangle (edge_triangle_intersect, contact.rs:324-352). A step
 * with self collision on runs the same scan at its committed positions. */
int mguso_scene_self_intersections(mguso_scene* s, const float* x, uint32_t* counts);

/* Assemble the Newton system once at positions x (f32[3 nv]) with inertia target x_tilde
   (f32[3 nv]; NULL means x), exactly as one Newton iteration of mguso_step does: contact
   stencils, elastic elements, colliders, contacts, right-hand side. The scene's positions
   are left at x. out3 = {blocks in the fixed pattern, contact-only blocks, stencils}.
   Parity and diagnostics entry; the reference counterpart is the triplet assembly of
   ImplicitSolver::step (core-engine/crates/engine-core/src/implicit.rs:2280-3155). */
int mguso_scene_assemble(mguso_scene* scene, const float* x, const float* x_tilde, uint32_t out3[3]);
/* The exact Hessian the adjoint's backward pass solves with, at x (no eigenvalue clamps; the
 * hinges' and barriers' second-derivative terms; each contact stiffness recorded from the
 * projected system at x, its mass part differentiated in the gap), assembled like
 * mguso_scene_assemble into the system mguso_scene_system downloads. */
int mguso_scene_assemble_exact(mguso_scene* scene, const float* x, const float* x_tilde, uint32_t out3[3]);

/* The step fraction the CCD filter allows for search direction dx (f32[3 nv]) from positions
   x (f32[3 nv]; the scene's positions are left at x): t_out f32[instances] (one per instance
   of a batch), cap_hits (optional) u32[instances] root solves that reached ccd_max_iter.
   Parity and diagnostics entry; counterpart: ImplicitSolver::ccd_max_step
   (core-engine/crates/engine-core/src/implicit.rs:1690-1947). */
int mguso_scene_ccd(mguso_scene* scene, const float* x, const float* dx, float* t_out, uint32_t* cap_hits);

/* Download the last assembled system: the fixed-pattern blocks (row_ptr u32[nv+1], col
   u32[out3[0]], values f32[9*out3[0]] row-major 3x3), the contact-only blocks in the same
   layout (out3[1] of them; col/val may be NULL when zero) and the right-hand side f32[3 nv].
   The system matrix is their sum. */
int mguso_scene_system(mguso_scene* scene, uint32_t* ps_row_ptr, uint32_t* ps_col, float* ps_val,
                       uint32_t* c_row_ptr, uint32_t* c_col, float* c_val, float* rhs);

/* The contact stencils of the last mguso_scene_assemble in assembly order: participants
   u32[4 n], kind u32[n] (0 vertex-triangle, 1 edge-edge) and gap f64[n]; min(n, cap) are
   written, *n_out = n. Counterpart: self_collision_stencils (implicit.rs:678-753). */
int mguso_scene_stencils(mguso_scene* scene, uint32_t cap, uint32_t* idx4, uint32_t* kind, double* d,
                         uint32_t* n_out);

#ifdef __cplusplus
}
#endif

#endif /* MGUSO_CUDA_H */
