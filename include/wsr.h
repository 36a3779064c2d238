/*
 * C ABI of the B200 WENO5-SR / WENO5-JS finite-volume path (libwsr.so).
 *
 * Plain pointers, sizes and an explicit CUDA stream (passed as void*; NULL = legacy default
 * stream). All array pointers are DEVICE pointers owned by the caller unless stated otherwise.
 * Every function returns an int status (WSR_OK = 0); wsr_last_error() gives the message.
 *
 * State layout: the reference's padded row-major array u[(ny+6)][(nx+6)][4] of FP64 conserved
 * variables (rho, rho u, rho v, E), ghost width 3 (warp_weno5_helpers.py:66-87). Ghost cells are
 * read through the boundary mapping and never written, exactly like the reference's stage buffers.
 *
 * Reference interfaces replaced (paths inside the reference project, code/snapshot/):
 *   wsr_closure_upload     load_mlp_params -> {w1..b4} device arrays
 *                          (run_weno5_circle_mlp_compare.py:49-81 FP64;
 *                           teacherfree_lab_weno5_mlp_f32/warp_mlp_f32/run_weno5_circle_mlp_compare_mlp_f32.py:52-84 FP32)
 *   wsr_euler2d_stage      launch_stage(u_stage, u0, u_out, stage, params, dt, rk, ...)
 *                          (for_paper_results/solvers/weno5_hllc.py:294-358 JS;
 *                           teacherfree_lab_weno5_v20_distance_balanced/weno5_hllc_refsym.py:298-435 SR FP64;
 *                           for_paper_results/solvers/weno5_hllc_mixed.py:121-168 SR FP32)
 *   wsr_euler2d_max_speed  compute_dt_from_warp_array's max-speed kernel (warp_weno5_helpers.py:189-207, 876-897)
 *   wsr_euler2d_run        run_to_time(initial, params, t_end, device, mlp_params, boundary, ...)
 *                          (weno5_hllc.py:386-410; weno5_hllc_refsym.py:462-544; weno5_hllc_mixed.py:185-212)
 */
#ifndef WSR_H
#define WSR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define WSR_OK 0
#define WSR_ERR_ARG 1         /* invalid argument (sizes, enum values, null pointers, short workspace) */
#define WSR_ERR_CUDA 2        /* a CUDA runtime call or kernel launch failed */
#define WSR_ERR_NO_CLOSURE 3  /* an SR method was requested before wsr_closure_upload */

/* methods: reconstruction weights and closure precision */
#define WSR_METHOD_JS 0       /* WENO5-JS, eps 1e-6, p 2 */
#define WSR_METHOD_SR_F64 1   /* WENO5-SR, FP64 MLP (REFSYM) */
#define WSR_METHOD_SR_F32 2   /* WENO5-SR, FP32 MLP, FP64 elsewhere (MIXED) */
#define WSR_METHOD_SR_BF16 3  /* WENO5-SR, BF16 inputs/parameters/activations, FP32 accumulation */
#define WSR_METHOD_Z 4        /* WENO-Z (Borges et al.): WENO5 p = 2, eps = h^2 of the reconstruction direction (2D,
                               * 3D, 1D scheme 5); WENO7 p = 3, eps = h^3 (1D scheme 7; the WENO7 2D functions
                               * document their own) */
#define WSR_METHOD_SR_BF16_TC 5 /* WENO5-SR with the BF16 closure's MLP on the tensor cores (warp mma.sync, BF16 x BF16
                                 * -> FP32); the same results as WSR_METHOD_SR_BF16 up to the accumulation order. An
                                 * addition without a counterpart in the reference; measured slower than
                                 * WSR_METHOD_SR_BF16 on B200, kept for that comparison. wsr_euler2d_stage(_at) and
                                 * wsr_euler2d_run only */

/* boundaries */
#define WSR_BC_TRANSMISSIVE 0
#define WSR_BC_PERIODIC 1
#define WSR_BC_DOUBLE_MACH 2 /* Mach-10 double-Mach reflection on [0, nx dx] x [0, ny dy] (time dependent;
                                 weno5_hllc_refsym.py:26-124); 2D stage and run functions only */
#define WSR_BC_Y_HALO 16     /* flag, OR-ed with WSR_BC_TRANSMISSIVE or WSR_BC_PERIODIC in wsr_euler2d_stage(_at):
                                the 3 ghost rows below and above the interior are read from the stage state as
                                stored (a slab of a y-decomposed grid whose halo the caller has exchanged); x ghosts
                                are derived from the base boundary as usual. wsr_euler2d_run rejects it. */

/* interface fluxes */
#define WSR_FLUX_HLLC 0
#define WSR_FLUX_FORCE 1

/* options bitmask */
#define WSR_OPT_ENO_CUTOFF 1  /* the reference's eno_cutoff flag (4e-7), off in all paper runs */
#define WSR_OPT_JS_FALLBACK 2 /* per-stencil WENO5-JS weights when the closure is non-finite, and per
                                 face when an SR face state has rho <= 0 or p <= 0 */
#define WSR_OPT_Z_HALO 8      /* wsr_euler3d_stage: the 3 z ghost planes below and above are filled by the caller
                                 (a slab of a z-decomposed grid) and not overwritten; x and y ghosts are filled as
                                 usual. wsr_euler3d_run rejects it. */
#define WSR_OPT_FACE_THREADS_8 32 /* 2D WENO5-SR stages (FP64, FP32, BF16 closures): eight threads per face in the
                                     two reconstruction kernels (16 faces per 128-thread block; each thread forms one
                                     stencil and at most one closure evaluation) whatever the grid size. By default
                                     SR stages use this form up to 128 x 128 cells, the four-thread form up to 256 x 256
                                     and one thread per face above (where one thread per face is no longer latency
                                     bound by its serial closure evaluations). Same results bit for bit in every form.
                                     JS, WENO-Z and the tensor-core closure always use one thread per face. */
#define WSR_OPT_FACE_THREADS_1 64 /* 2D WENO5 stages: one thread per face whatever the grid size */
#define WSR_OPT_FACE_THREADS_4 128 /* 2D WENO5-SR stages: four threads per face (32 faces per block, two stencils each)
                                      whatever the grid size */

typedef struct wsr_ctx wsr_ctx;

/* Create a context bound to CUDA device `device`. */
int wsr_ctx_create(int device, wsr_ctx **out);
void wsr_ctx_destroy(wsr_ctx *ctx);
/* Message of the last failed call on this context (static storage inside the context). With a null context: the
 * message of the last wsr_ctx_create that failed on the calling thread (thread-local storage), e.g. no CUDA device. */
const char *wsr_last_error(const wsr_ctx *ctx);

/* Closure parameters: `packed` is a HOST array in the order w1 b1 w2 b2 w3 b3 w4 b4 ([in][out]
 * row-major, the .npz arrays without their leading dimension): kind 5 (WENO5, 5->10->6->6->3) takes
 * n = 189 values, kind 7 (WENO7, 6->24->16->16->4) n = 908. The FP64, FP32 and BF16 methods use the
 * values rounded to their precision. */
int wsr_closure_upload(wsr_ctx *ctx, int kind, const double *packed, int n);

/* ---- 2D Euler WENO7 with Shu's fourth-order TVD Runge-Kutta (weno7_point_rk4_shu/point_rk4.py) ----
 * State: padded [ny+8][nx+8][4] FP64 conserved (ghost width 4); characteristic WENO7 normal reconstruction,
 * conservative two-point Gauss WENO7 transverse reconstruction, HLLC; boundary WSR_BC_TRANSMISSIVE or
 * WSR_BC_PERIODIC (ghost cells are derived, never read from u). */
size_t wsr_euler2d_w7_workspace_bytes(int nx, int ny);
/* One right-hand side into rhs (interior [ny][nx][4]): L(u) (reverse = 0) or the downwind operator L~(u)
 * whose interface fluxes take the Gauss states in swapped order (reverse = 1); compute_rhs of
 * point_rk4.py:435-511. method: WSR_METHOD_JS (classical weights), WSR_METHOD_Z (WENO-Z, p = 3, betas / 240,
 * eps = dx^3 along x and dy^3 along y: weno_z_borges_p2_results/weno7_point_rk4_z.py, weight_kind 1) or
 * WSR_METHOD_SR_F64 (betas of the FP64 WENO7 closure uploaded with wsr_closure_upload(ctx, 7, ...), the lr = 2
 * face and the second Gauss point from the flipped stencil; compute_rhs_mlp of
 * teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/point_rk4_mlp.py:198-277 with eno_cutoff off).
 * WSR_METHOD_SR_F64 without an uploaded WENO7 closure returns WSR_ERR_NO_CLOSURE.
 * opts: 0, or WSR_OPT_JS_FALLBACK with WSR_METHOD_SR_F64 (an addition; the reference stops the run instead): a
 * stencil whose closure betas are not finite takes WENO7-JS weights, and a normal face state with rho <= 0 or
 * p <= 0 is recomputed with WENO7-JS weights; both are counted (wsr_euler2d_w7_counters, out_host[4]). */
int wsr_euler2d_w7_rhs(wsr_ctx *ctx, const double *u, double *rhs, int nx, int ny, double dx, double dy,
                       double gamma, int bc, int method, int reverse, int opts, void *workspace,
                       size_t workspace_bytes, void *stream);
/* Time loop of run_from_initial (point_rk4.py:568-600) on u in place from time t_start: dt = cfl min(dx, dy)
 * / max speed, the loop runs while t < t_end, a step that would pass t_end is shortened to reach it; at most
 * max_steps steps. dts_host (capacity max_steps) receives each step's dt. */
int wsr_euler2d_w7_run(wsr_ctx *ctx, double *u, int nx, int ny, double dx, double dy, double gamma, double cfl,
                       double t_start, double t_end, int bc, int method, int opts, int max_steps, double *dts_host,
                       int *steps_out, double *t_out, void *workspace, size_t workspace_bytes, void *stream);
/* WSR_METHOD_SR_F64 closure evaluations (stencils that ran the MLP pair) since the last wsr_euler2d_w7_rhs /
 * wsr_euler2d_w7_run on this workspace: out_host[0..3] = normal x, normal y, transverse x, transverse y;
 * out_host[4] = JS fallbacks taken under WSR_OPT_JS_FALLBACK (out_host holds 5 values). Synchronous. */
int wsr_euler2d_w7_counters(wsr_ctx *ctx, void *workspace, size_t workspace_bytes, int nx, int ny,
                            unsigned long long *out_host);

/* Bytes of device workspace the 2D functions need for an nx x ny interior. */
size_t wsr_euler2d_workspace_bytes(int nx, int ny);

/* One SSPRK3 stage (rk = 1, 2, 3): writes the interior of u_out from u_stage and u0
 * (rk 1: rhs; rk 2: 3/4 u0 + 1/4 rhs; rk 3: 1/3 u0 + 2/3 rhs). dt is a host value. */
int wsr_euler2d_stage(wsr_ctx *ctx, const double *u_stage, const double *u0, double *u_out, int nx, int ny,
                      double dx, double dy, double gamma, double dt, int rk, int method, int bc, int flux,
                      int opts, void *workspace, size_t workspace_bytes, void *stream);

/* wsr_euler2d_stage with the boundary evaluated at boundary_time (the reference's launch_stage
 * boundary_time argument, weno5_hllc_refsym.py:298-311); only the double-Mach boundary depends on it.
 * wsr_euler2d_run uses t, t + dt and t + dt/2 for the three stages of a step. */
int wsr_euler2d_stage_at(wsr_ctx *ctx, const double *u_stage, const double *u0, double *u_out, int nx, int ny,
                         double dx, double dy, double gamma, double dt, int rk, int method, int bc, int flux,
                         int opts, double boundary_time, void *workspace, size_t workspace_bytes, void *stream);

/* max over the interior of max(|u|+c, |v|+c), rho and p floored at 1e-15. Synchronises `stream`
 * and writes the host value. */
int wsr_euler2d_max_speed(wsr_ctx *ctx, const double *u, int nx, int ny, double gamma, double *out_host,
                          void *workspace, size_t workspace_bytes, void *stream);

/* Time loop of run_to_time with dt, t and the stop test kept on the device.
 * u[4] are four padded state buffers: u[0] holds the initial state on entry, u[1], u[2] are stage
 * buffers, u[3] the swap partner of u[0]. Step s advances from u[0] to u[3] when s is even and from
 * u[3] to u[0] when it is odd; *final_slot (0 or 3) says which holds the result.
 * The loop starts at time t_start (0 for a fresh run; a resumed run passes the time reached).
 * t_end: stop when t >= t_end - 1e-14 (the last dt is clipped). fixed_steps > 0 instead runs exactly
 * that many full CFL steps. check_health != 0 stops after step 1 (and every check_interval steps when
 * check_interval > 0) if the state holds a NaN or p <= 0. dts_host (capacity max_steps) receives each
 * step's dt; the loop also stops at max_steps. */
int wsr_euler2d_run(wsr_ctx *ctx, double *const u[4], int nx, int ny, double dx, double dy, double gamma,
                    double cfl, double t_start, double t_end, int method, int bc, int flux, int opts, int check_health,
                    int check_interval, int fixed_steps, int max_steps, double *dts_host, int *steps_out,
                    double *t_out, int *final_slot, int *fallbacks_out, void *workspace, size_t workspace_bytes,
                    void *stream);

/* ---- host-buffer steps (the reference's drivers keep the state in host arrays) ----
 * Copies the interior of u_host (a padded [ny+6][nx+6][4] HOST array; pinned memory for overlap) into u[0],
 * advances `steps` full CFL steps exactly as wsr_euler2d_run with fixed_steps does (same buffers, same results bit
 * for bit), and copies the result's interior back into u_host; the ghost cells of u_host are not touched. The
 * copies run on the context's own copy streams in `bands` row bands (0: one per 250 rows, at most 16, the first
 * and last half as high; pageable memory: one band):
 *   - the first stage's wave speed and, under WSR_BC_TRANSMISSIVE, its normal reconstructions start on each
 *     band as it arrives;
 *   - the last stage runs band by band and each band's read-back starts as soon as its rows are final.
 * flags 0: returns when u_host holds the result. WSR_HOST_ASYNC: returns once everything is queued. A following
 * call on the same host array and device buffers uploads band k right after this call's read-back of band k, so
 * consecutive calls overlap both copy directions with the computation; between such calls u[0..3] belong to the
 * pipeline (wsr_euler2d_stage(_at) and wsr_euler2d_run on the same context order their work after the read-backs
 * still in flight, as wsr_euler2d_host_order does). wsr_euler2d_host_order makes `stream` wait for the read-backs;
 * wsr_euler2d_host_wait synchronises, reports the steps taken and JS fallbacks summed over the calls since the
 * previous wait, and returns an error that any of them met on the device. */
#define WSR_HOST_ASYNC 1
int wsr_euler2d_advance_host(wsr_ctx *ctx, double *u_host, double *const u[4], int nx, int ny, double dx, double dy,
                             double gamma, double cfl, int steps, int method, int bc, int flux, int opts, int flags,
                             int bands, void *workspace, size_t workspace_bytes, void *stream);
int wsr_euler2d_host_order(wsr_ctx *ctx, void *stream);
int wsr_euler2d_host_wait(wsr_ctx *ctx, int *steps_out, int *fallbacks_out);

/* ---- batched 1D periodic linear advection u_t + a u_x = 0 ----
 * Replaces the reference's torch steppers (teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/
 * rk3_advection.py:118-186 ssprk3_step_signed / rollout_distance; teacherfree_lab_weno7_rk4_distance_
 * balanced_fast/rk4_advection.py:137-220 shu_rk4_step_signed / rollout_signed; for_paper_results/
 * run_gste.py:103-118 integrate_ssprk3) for a ragged batch of B independent trajectories packed in u:
 * trajectory b occupies u[offsets[b] .. offsets[b+1]) (n_b cells on a periodic grid of spacing dx[b]),
 * advects with velocity[b] (its sign picks the upwind side), and takes n_full[b] steps of dt_full[b]
 * followed, when dt_last[b] > 0, by one step of dt_last[b] (the reference's CFL schedule; the GSTE
 * schedule is n_full steps of t/n_full). u is updated in place. order (optional, B entries) is the
 * visiting order of trajectories (longest first balances the launch). nmax >= every n_b, at most 2048.
 * scheme 5: WENO5 (5-point stencils, closure kind 5); scheme 7: WENO7 (7-point stencils, closure kind 7).
 * method WSR_METHOD_Z gives the WENO-Z baselines of weno_z_borges_p2_results/torch_weno_z.py:14-107 (WENO5-Z:
 * tau5 = |b0 - b2|, eps = dx[b]^2, p = 2; WENO7-Z: tau7 = |-b0 - 3 b1 + 3 b2 + b3|, eps = dx[b]^3, p = 3).
 * All array arguments are device pointers. fallbacks_out, errors_out and counters_out (2 values: MLP
 * evaluations, plateau stencils when opts has WSR_OPT_COUNT) are host pointers or NULL; when any is
 * given the call synchronises `stream`. */
#define WSR_INTEG_SSPRK3 0
#define WSR_INTEG_SHU_RK4 1
size_t wsr_adv1d_workspace_bytes(void);
int wsr_adv1d_run(wsr_ctx *ctx, double *u, const long long *offsets, const int *order, const double *velocity,
                  const double *dx, const int *n_full, const double *dt_full, const double *dt_last, int B, int nmax,
                  int scheme, int method, int integrator, int opts, int *fallbacks_out, int *errors_out,
                  unsigned long long *counters_out, void *workspace, size_t workspace_bytes, void *stream);

/* ---- closure training through 1D advection trajectories (WENO5-SR + SSPRK3) ----
 * Replaces the reference's autograd training objective (teacherfree_lab_weno5_v20_distance_balanced_
 * mlp_f32_fast/fast_losses.py:412-648 fast_autoregressive_trajectory_loss and its loss.backward(),
 * called from train.py:474-520) with the plain L1 loss
 *     L = sum_{b, k = 1..steps, i} |u_{b,k,i} - e_{b,k,i}| / (B * steps * n)
 * of B periodic trajectories of n cells (u0: B x n, row-major, device; NULL starts every trajectory from the
 * exact cell averages of its profile), velocity[b] = +1 or -1, each taking
 * `steps` SSPRK3 steps of dt on a grid of spacing dx, against the exact cell averages e of the advected
 * profile desc[b] (B x WSR_PROFILE_LEN, device; layout of weno_sr_publishing_b200/profiles.py).
 * method: WSR_METHOD_SR_F64 or WSR_METHOD_SR_F32 with the WENO5 closure of wsr_closure_upload.
 * wsr_train1d_forward writes the loss to loss_out (1 double, device), the final states to u_final (B x n,
 * device, or NULL), and keeps in the workspace the states of every ckpt_every-th step and the signs of
 * u - e. wsr_train1d_backward then writes dL/dtheta (189 doubles, packed w1 b1 .. b4, device) to grad_out
 * and, when grad_u0 is not NULL, dL/du0 (B x n, device): a hand-written adjoint that recomputes one
 * checkpoint segment at a time. The backward call takes the same arguments and workspace as the forward
 * call before it, with the closure unchanged in between. n <= 1024. The result is deterministic. */
#define WSR_PROFILE_LEN 34
size_t wsr_train1d_workspace_bytes(int B, int n, int steps, int ckpt_every);
int wsr_train1d_forward(wsr_ctx *ctx, const double *u0, const double *desc, const double *velocity, int B, int n,
                        double dx, double dt, int steps, int ckpt_every, int method, double *loss_out,
                        double *u_final, void *workspace, size_t workspace_bytes, void *stream);
int wsr_train1d_backward(wsr_ctx *ctx, const double *velocity, int B, int n, double dx, double dt, int steps,
                         int ckpt_every, int method, double *grad_out, double *grad_u0, void *workspace,
                         size_t workspace_bytes, void *stream);

/* ---- 3D Euler, WENO5 (JS / SR / Z) with 2 x 2 Gauss-point transverse quadrature ----
 * Replaces the reference's 3D Warp port (warp_weno5_3d_rk3/solver.py:165-329 Weno5Rk3Solver: _rk_stage,
 * advance; kernels.py:776-1163) and its WENO-Z variant (weno_z_borges_p2_results/weno5_3d_solver_z.py,
 * weno5_3d_kernels_z.py: method WSR_METHOD_Z, eps = h^2 of each reconstruction's direction). State layout: padded row-major q[nz+6][ny+6][nx+6][5] doubles, conserved
 * (rho, rho u, rho v, rho w, E), ghost width 3, gamma 1.4 (config.py:45-52). Boundaries are transmissive;
 * `inflow` (a HOST array of 5 conserved values, or NULL) instead fixes the x-low ghost cells.
 * flux: WSR_FLUX3_EVILIN (the reference's interface state) or WSR_FLUX3_HLLC (HLLC in 3D, an addition).
 * wsr_euler3d_stage runs one RK stage in place (stage 1 also saves the stage-start state in the workspace,
 * which stages 2 and 3 use), with dt a host value. wsr_euler3d_run advances up to max_steps steps with dt
 * = cfl min(dx, dy, dz) / max speed (1e10 below 1e-15) kept on the device, stopping at t_end (pass a huge
 * t_end for a fixed number of steps); dts_host (capacity max_steps, or NULL) receives each step's dt. */
#define WSR_FLUX3_EVILIN 0
#define WSR_FLUX3_HLLC 1
size_t wsr_euler3d_workspace_bytes(int nx, int ny, int nz);
int wsr_euler3d_stage(wsr_ctx *ctx, double *q, int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                      int stage, int method, int flux, int opts, const double *inflow, void *workspace,
                      size_t workspace_bytes, void *stream);
int wsr_euler3d_max_speed(wsr_ctx *ctx, const double *q, int nx, int ny, int nz, double *out_host, void *workspace,
                          size_t workspace_bytes, void *stream);
int wsr_euler3d_run(wsr_ctx *ctx, double *q, int nx, int ny, int nz, double dx, double dy, double dz, double cfl,
                    double t_start, double t_end, int max_steps, int method, int flux, int opts, const double *inflow,
                    double *dts_host, int *steps_out, double *t_out, void *workspace, size_t workspace_bytes,
                    void *stream);
/* Closure tallies of the last 3D stage/run made with WSR_OPT_COUNT: out_host[0..5] = (MLP, plateau) stencils
 * of the normal, first transverse and second transverse (flux) kernels; out_host[6] = JS fallbacks taken under
 * WSR_OPT_JS_FALLBACK (stencils whose closure output is not finite, and normal face states with rho <= 0 or
 * p <= 0 recomputed with WENO5-JS weights; an addition without a counterpart in the reference). out_host holds
 * 7 values. */
int wsr_euler3d_counters(wsr_ctx *ctx, void *workspace, size_t workspace_bytes, int nx, int ny, int nz,
                         unsigned long long *out_host);

/* ---- measurement hooks (no counterpart in the reference, which times whole runs with
 * time.perf_counter in for_paper_results/run_weno5_timing.py:111-140) ---- */

/* Kernel classes reported by wsr_profile_read. */
#define WSR_PROF_NORMAL_X 0
#define WSR_PROF_NORMAL_Y 1
#define WSR_PROF_FLUX_X 2
#define WSR_PROF_FLUX_Y 3
#define WSR_PROF_UPDATE 4
#define WSR_PROF_CONTROL 5
#define WSR_PROF_KINDS 6

/* Bracket every kernel launched through this context with CUDA events on its stream (on != 0), and
 * reset the totals. */
int wsr_profile_enable(wsr_ctx *ctx, int on);
/* Synchronise the recorded events and return, per kernel class, the summed device time in ms and the
 * launch count (arrays of WSR_PROF_KINDS). */
int wsr_profile_read(wsr_ctx *ctx, double *ms, long long *launches);

/* ---- device-resident time loop of one y-slab (an addition: the reference runs one grid per GPU) ----
 * The dt rule, the stop test and t live in the workspace's control block, as in wsr_euler2d_run, so a decomposed
 * run needs no host synchronisation per step. Per step, on the slab's stream:
 *   wsr_euler2d_slab_step(phase 0)   dt from the wave-speed slot (which must hold the MAX over all slabs), the stop
 *                                    test, the slot cleared for the step's own maximum;
 *   3 x (halo exchange by the caller, WSR_BC_Y_HALO rows; wsr_euler2d_slab_stage(rk = 1, 2, 3))  the SSPRK3 stages
 *                                    with the control block's dt; the third leaves the local wave speed in the slot;
 *   all-reduce (MAX) of the slot across ranks by the caller (the slot holds the non-negative double's bit pattern,
 *                                    so a 64-bit integer MAX is the MAX of the speeds);
 *   wsr_euler2d_slab_step(phase 1)   t += dt, steps += 1.
 * wsr_euler2d_slab_begin initialises the control block and puts the initial state's local wave speed in the slot
 * (all-reduce it before the first step); wsr_euler2d_slab_speed_slot returns the slot's device address;
 * wsr_euler2d_slab_status synchronises the stream and reads steps, t, the stop flag and the ring of the last 64 dts
 * (dts_ring[s % 64] = dt of step s). Steps launched after the stop flag is set do nothing, so the caller may launch
 * several steps between status reads; the result is in the buffer of step `steps`. */
int wsr_euler2d_slab_begin(wsr_ctx *ctx, const double *u, int nx, int ny, double dx, double dy, double gamma,
                           double cfl, double t_start, double t_end, int max_steps, void *workspace,
                           size_t workspace_bytes, void *stream);
int wsr_euler2d_slab_speed_slot(wsr_ctx *ctx, void *workspace, size_t workspace_bytes, int nx, int ny,
                                unsigned long long **slot);
int wsr_euler2d_slab_step(wsr_ctx *ctx, int phase, int nx, int ny, double dx, double dy, void *workspace,
                          size_t workspace_bytes, void *stream);
int wsr_euler2d_slab_stage(wsr_ctx *ctx, const double *u_stage, const double *u0, double *u_out, int nx, int ny,
                           double dx, double dy, double gamma, int rk, int method, int bc, int flux, int opts,
                           void *workspace, size_t workspace_bytes, void *stream);
int wsr_euler2d_slab_status(wsr_ctx *ctx, void *workspace, size_t workspace_bytes, int nx, int ny, int *steps,
                            double *t, int *done, double *dts_ring, void *stream);

/* Closure tallies of the last run/stage made with WSR_OPT_COUNT, per kernel class k = normal x,
 * normal y, flux x, flux y: out_host[2k] = stencils that ran the MLP pair, out_host[2k+1] = plateau
 * stencils that took the linear weights (out_host holds 8 values). */
#define WSR_OPT_COUNT 4
int wsr_euler2d_counters(wsr_ctx *ctx, void *workspace, size_t workspace_bytes, int nx, int ny,
                         unsigned long long *out_host);

/* Measured FMA throughput of this GPU in TFLOP/s (bits = 32 or 64; 2 flops per FMA). */
int wsr_probe_peak_flops(wsr_ctx *ctx, int bits, double *tflops, void *stream);
/* The table-driven FP64 exponential of the WENO7-SR closure on n device values (out[i] = exp(x[i]), arguments
 * clamped to [-700, 700]); for checking it against the CUDA math library. */
int wsr_probe_exp_tab(wsr_ctx *ctx, const double *x, double *out, int n, void *stream);

/* ---- stage without any allocation (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc (a host that owns all device memory through its own pool,
 * or a step that must not pay cudaMalloc's implicit synchronisation). One SSPRK3 stage like
 * wsr_euler2d_stage, with its scratch in a static device array of WSR_NOALLOC_SCRATCH_BYTES (32 MiB,
 * enough for grids up to 400 x 400) that every GPU loading the library holds until exit.
 * Supported: method WSR_METHOD_JS, WSR_METHOD_Z, WSR_METHOD_SR_F64, WSR_METHOD_SR_F32 or WSR_METHOD_SR_BF16;
 * bc WSR_BC_TRANSMISSIVE or WSR_BC_PERIODIC (no double-Mach boundary, no WSR_BC_Y_HALO); flux WSR_FLUX_HLLC or
 * WSR_FLUX_FORCE. Anything else returns WSR_ERR_ARG.
 * No context: `closure_params` is a HOST array of the 189 packed parameters (NULL for WSR_METHOD_JS and
 * WSR_METHOD_Z). Runs on the calling thread's current device; `stream` must belong to it. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and must come before any stream capture on
 * that device; the address is cached for the process and is not valid after cudaDeviceReset. On entry the
 * call clears this thread's pending CUDA launch error (cudaGetLastError), so that WSR_ERR_CUDA reports its own
 * launches. Grids whose workspace exceeds the array return WSR_ERR_SCRATCH_LIMIT. All calls on a device share
 * the array: calls that overlap on the GPU race and must be serialised by the caller.
 * Returns status codes only (no message). */
#define WSR_ERR_SCRATCH_LIMIT 4
#define WSR_NOALLOC_SCRATCH_BYTES (32u << 20)
int wsr_euler2d_stage_noalloc(const double *u_stage, const double *u0, double *u_out, int nx, int ny, double dx,
                              double dy, double gamma, double dt, int rk, int method, int bc, int flux, int opts,
                              const double *closure_params, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* WSR_H */
