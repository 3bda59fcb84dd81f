/*
 * cgli_fu_flow.h -- C ABI of the B200 implementation of the CGLI_Fu_Flow
 * per-step hot path (MUSCL-5 / preconditioned Roe fluxes, viscous terms,
 * BDF2 dual-time residual, two symmetric LU-SGS i+j+k wavefront sweeps,
 * primitive update and residual norms, wall / periodic boundaries and the
 * driving force), on one GPU.
 *
 * Conventions shared by every entry point:
 *   - plain C types only; every call returns 0 on success and a negative
 *     CGLI_E* code on failure, with a message from cgli_last_error();
 *   - the caller owns host buffers; the library owns device memory, one CUDA
 *     stream per context; a context is not thread-safe;
 *   - host arrays use the reference layout of Array.h:7-186: one contiguous
 *     double array per field, [X_np][Y_m][Z_m] with k fastest, X_np = Nx+6,
 *     Y_m = Ny+4, Z_m = Nz+4, conserved variables stored as Q/J; face arrays
 *     keep the reference's shifted indexing (x-face i+1/2 of cell (i,j,k) at
 *     [i][j-1][k-1], y-face at [i-1][j][k-1], z-face at [i-1][j-1][k]);
 *   - the x direction is periodic: the reference's MPI slab halos
 *     (main.cpp:167-200, Dual_time_stepping.cpp:942-976) become a copy of the
 *     slab's own far planes, with the same one-iteration lag.
 */
#ifndef CGLI_FU_FLOW_H
#define CGLI_FU_FLOW_H

#ifdef __cplusplus
extern "C" {
#endif

#define CGLI_OK 0
#define CGLI_EINVAL (-1)      /* bad argument / unknown array name / size out of range */
#define CGLI_ECUDA (-2)       /* CUDA runtime error */
#define CGLI_ENOMEM (-3)      /* device allocation failed */
#define CGLI_ESTATE (-4)      /* call order violated (e.g. no metrics yet) */
#define CGLI_EDIVERGED (-5)   /* residual norm not finite */
#define CGLI_ETIMEOUT (-6)    /* a device-side wait gave up (wavefront flag) */

#define CGLI_FP64 0           /* everything in double precision */
#define CGLI_MIXED 1          /* LU-SGS sweeps, split Jacobians, diagonal in float */

/* Runtime replacement of the compile-time parameters of Resolution.h,
 * prm.h and Viscous_terms.h, plus the run constants main.cpp:44-70 fixes. */
typedef struct cgli_params {
  int nx, ny, nz;          /* interior cells (X_out of one slab, Y_out, Z_out) */
  double dxi, det, dzt;    /* deltaXI, deltaET, deltaZT (Resolution.h:19-21) */
  double dt;               /* physical time step deltaT (main.cpp:58) */
  double e;                /* preconditioning floor e (main.cpp:57) */
  double mu, pr;           /* mu_L, Pr_L (Viscous_terms.h:4-5) */
  double twall_lo, twall_hi; /* wall temperatures (Y_boundary_condition.cpp:139,166) */
  double force;            /* uniform x body force (replaces Dual_time_stepping.cpp:831) */
  int precision;           /* CGLI_FP64 or CGLI_MIXED */
  int curved_walls;        /* 0: the wall-face flux of Flux_Y.cpp:400-408 (flat walls);
                            * 1: plus the x and z components of the wall pressure
                            * force, 0.5 (eta_x, eta_z) (p_L + p_R) / J_v, which
                            * flat walls do not have (identical for flat walls) */
  int x_open;              /* 0: one slab of the x-periodic channel (the workloads);
                            * 1: the reference's open configuration run as a single
                            * rank 0 of 1: characteristic inflow / outflow ghost planes
                            * (cgli_x_boundary_condition), one-sided MUSCL at the x ends
                            * (Flux_X.cpp:139-216), no x halo, zero implicit halos
                            * (Dual_time_stepping.cpp:204-246), end-plane metrics of
                            * Jacobian.cpp:110-157 from cgli_channel_metrics */
  int nx_inlet, nx_outlet; /* sponge layers of Resolution.h:5-6 (x_open only; the
                            * residual of Dual_time_stepping.cpp:554-664); the walls are
                            * isothermal only between them (Y_boundary_condition.cpp:114) */
  int buoyancy;            /* 1: body force f = -(rho - 1.1842) 9.81 per cell
                            * (Dual_time_stepping.cpp:831) instead of `force` (the DP-LUR
                            * solver keeps `force` and has no sponge, as DPLUSGS.cpp) */
  double high;             /* channel height of prm.h:16 (sponge strength
                            * Sigma = Sigma_0 U / high); needed with sponge layers */
} cgli_params;

typedef struct cgli_ctx cgli_ctx;

/* ---- lifecycle (replaces Array.h allocation and main.cpp:19-141 set-up) */
int cgli_create(const cgli_params *p, cgli_ctx **out);
int cgli_destroy(cgli_ctx *ctx);
const char *cgli_last_error(void);
/* device bytes the context holds */
long long cgli_device_bytes(const cgli_ctx *ctx);

/* ---- array transfer by reference name ("U1_".."U5_", "U1".."U5", "U1q".."U5q",
 * "J", "xidx".."ztdz", the same with "_u"/"_v"/"_w" and "J_u"/"J_v"/"J_w",
 * "inFx1".."inFz5", "vF2".."vF5", "MR1".."MR5", "NR1".."NR5", "EpX"/"EpY"/"EpZ",
 * "Y_point").  Each transfers X_np*Y_m*Z_m doubles. */
int cgli_set_array(cgli_ctx *ctx, const char *name, const double *host);
int cgli_get_array(cgli_ctx *ctx, const char *name, double *host);

/* Analytic channel metrics of Jacobian.cpp:61-243, Jacobian_u.cpp:59-101,
 * Jacobian_v.cpp:79-151, Jacobian_w.cpp:61-106 (tanh wall clustering with
 * parameter `stretch`, channel height `high`), generated on the host and
 * uploaded; bit-identical to the reference's arrays, ghost-row copy typos
 * included. */
int cgli_channel_metrics(cgli_ctx *ctx, double high, double stretch);
/* The same generator on the host only (no device, no context): writes the
 * one metric array `name` ("J", "xidx".."ztdz", "J_u", "etdy_v", ...) of an
 * Nx x Ny x Nz slab into `out` (X_np*Y_m*Z_m doubles). */
int cgli_channel_metrics_host(int nx, int ny, int nz, double det, double high, double stretch,
                              const char *name, double *out);
/* Curvilinear metrics of a channel with a wavy lower wall (no reference
 * code: the workload that exercises every metric term).  Mapping x = xi,
 * z = zeta, y = yw(x) + (high - yw(x)) Y0(eta) / high with the tanh
 * clustering Y0 of cgli_channel_metrics and yw(x) = amplitude sin(4 pi x /
 * Lx), Lx = Nx * deltaXI; J = 1 / y_eta, etdx = -y_xi / y_eta,
 * etdy = 1 / y_eta, xidx = ztdz = 1, other terms zero, at the cell and face
 * positions and with the ghost rules of the channel generator.
 * |amplitude| < high / 2. */
int cgli_wavy_channel_metrics(cgli_ctx *ctx, double high, double stretch, double amplitude);
int cgli_wavy_channel_metrics_host(int nx, int ny, int nz, double dxi, double det, double high, double stretch,
                                   double amplitude, const char *name, double *out);

/* Sets Q^(n+1,m) (U_), Q^n (U) and Q^(n-1) (Uq), 5 arrays each, in the
 * reference layout (Initial_condition.cpp:111-236 and main.cpp:127-141). */
int cgli_set_state(cgli_ctx *ctx, const double *const U_[5], const double *const U[5],
                   const double *const Uq[5]);
/* Reads back Q^(n+1,m) (5 arrays). */
int cgli_get_state(cgli_ctx *ctx, double *const U_[5]);
/* The time levels of the next step from a host-driven loop that keeps them
 * itself (it does main.cpp:364-386 on the host): U_ = U = U[v] (Q^n/J) and
 * Uq = Uq[v] (Q^(n-1)/J), reference layout.  Q^n crosses the bus once (U_ is
 * a device copy), and the previous device Uq becomes Q^(n-2) of the
 * extrapolated guess.  Unlike cgli_set_state, the running maxima of the
 * stopping rule and the step history carry on. */
int cgli_set_levels(cgli_ctx *ctx, const double *const U[5], const double *const Uq[5]);
/* ---- restart files in the reference's format.  cgli_write_restart writes
 * Q^n = U*J and Q^(n-1) = Uq*J of this slab into `path` as Output.cpp:187-284
 * lays out LES%05d.bin: ten fields, each spanning a global x extent of
 * global_nx planes, this slab at planes [x_offset, x_offset + Nx), k fastest
 * (single GPU: global_nx = Nx, x_offset = 0; one slab of a multi-slab file
 * otherwise, the file is not truncated).  cgli_read_restart reads such a file
 * as Initial_condition.cpp:56-236 does (quiescent state on the interior
 * planes, then the slab's cells as Q/J; U_ = U) and acts as cgli_set_state.
 * The metrics must be set first.  cgli_write_history / cgli_read_history keep
 * what the reference format has no room for (no counterpart in the
 * reference): the raw levels U_, U, Uq and Q^(n-2)/J with their ghost cells,
 * the driving force, the running maxima of the norms and the step history;
 * reading the sidecar after the file continues the run bit for bit (the
 * file alone loses the lagged ghost values and the rounding of Q = U*J). */
int cgli_write_restart(cgli_ctx *ctx, const char *path, int global_nx, int x_offset);
int cgli_read_restart(cgli_ctx *ctx, const char *path, int global_nx, int x_offset);
int cgli_write_history(cgli_ctx *ctx, const char *path);
int cgli_read_history(cgli_ctx *ctx, const char *path);

/* Copies the time levels (U_, U, Uq, Q^(n-2)), the driving force, the
 * running maxima of the norms and the step history of `src` into `dst`
 * (device to device; same grid, any precision), so that several contexts
 * continue one run from the same point. */
int cgli_copy_state(cgli_ctx *dst, const cgli_ctx *src);

/* ---- the reference routines, one entry point each, acting on the device state */
/* main.cpp:167-200: periodic 3-plane halo of U_ in x */
int cgli_halo_x(cgli_ctx *ctx);
/* Y_boundary_condition.cpp:19-186 (replaces Y_boundary_condition()) */
int cgli_y_boundary_condition(cgli_ctx *ctx);
/* Z_boundary_condition.cpp:15-69 (replaces Z_boundary_condition()) */
int cgli_z_boundary_condition(cgli_ctx *ctx);
/* Flux_X.cpp:12-359, Flux_Y.cpp:15-415, Flux_Z.cpp:15-360: fill inFx/inFy/inFz */
int cgli_flux_x(cgli_ctx *ctx);
int cgli_flux_y(cgli_ctx *ctx);
int cgli_flux_z(cgli_ctx *ctx);
/* X_boundary_condition.cpp:73-338 (x_open): one pseudo-time step of the
 * characteristic inflow / outflow relations on ghost planes 2 and Nx+3;
 * no-op for the periodic slab, like the reference's interior ranks.
 * cgli_halo_x is a no-op on an open slab (both neighbours absent). */
int cgli_x_boundary_condition(cgli_ctx *ctx);
/* Viscous_terms.cpp:15-907: fill vF2..vF5 */
int cgli_viscous_terms(cgli_ctx *ctx);
/* Dual_time_stepping.cpp:18-1795: residual, 2 x (forward + backward)
 * hyperplane sweeps, update of U_, five norms er[v] = sqrt(sum)/(Nx Ny Nz)
 * (the reference divides by its global X_out). Reads the inF and vF arrays
 * filled by the three flux entry points and cgli_viscous_terms. */
int cgli_dual_time_stepping(cgli_ctx *ctx, double er[5]);

/* DPLUSGS.cpp:18-1240, the DP-LUR alternative to Dual_time_stepping that
 * main.cpp:268-284 leaves commented out: the same residual, four Jacobi
 * relaxations of the same split-Jacobian operator (inviscid diagonal), the
 * update of U_, five norms er[v] = sqrt(sum of r_v^2)/(Nx Ny Nz) with r the
 * squared increments of p, u, v, w, T (the reference divides by its global
 * X_out).  Needs precision CGLI_FP64. */
int cgli_dplusgs(cgli_ctx *ctx, double er[5]);

#define CGLI_LUSGS 0          /* inner solver: Dual_time_stepping's LU-SGS sweeps */
#define CGLI_DPLUR 1          /* inner solver: DPLUSGS's Jacobi relaxations */
/* Inner solver of cgli_inner_iteration and cgli_step: the reference's
 * Dual_time_stepping call (main.cpp:245-262, the default) or its commented
 * DPLUSGS call (main.cpp:268-284).  CGLI_DPLUR needs precision CGLI_FP64. */
int cgli_set_inner_solver(cgli_ctx *ctx, int solver);

/* One complete inner iteration (main.cpp:167-264) through the fused fast
 * path: halo + boundaries, fluxes, viscous terms, the dual-time residual,
 * then the wavefront sweeps and the update (CGLI_LUSGS) or the relaxations
 * and the update (CGLI_DPLUR). */
int cgli_inner_iteration(cgli_ctx *ctx, double er[5]);

/* Driven_force.cpp:14-74: bulk mass flux (volume-weighted mean of rho*u) */
int cgli_driven_force(cgli_ctx *ctx, double *bulk_flux);
/* main.cpp:364-386: Q^(n-1) <- Q^n, Q^n <- Q^(n+1) */
int cgli_end_step(cgli_ctx *ctx);
/* uniform driving force used by the next residual assembly */
int cgli_set_force(cgli_ctx *ctx, double force);

/* One physical step (main.cpp:157-386): the initial guess of the chosen
 * predictor, inner iterations until every one of the five norms divided by
 * its running maximum over the run (main.cpp:287-297, reset by
 * cgli_set_state) is below `drop`, or `cap` iterations ran (fixed_iters > 0
 * runs exactly that many), then the time-level shift (Q^(n-2) is kept too).
 * Returns the iteration count and the final norms. */
int cgli_step(cgli_ctx *ctx, int fixed_iters, double drop, int cap, int *iters, double er[5]);
/* The five norms of every inner iteration of the last cgli_step, iteration
 * by iteration (norms[5*i + v]); copies min(iterations, max_iters) rows and
 * returns the iteration count in *iters. */
int cgli_step_norms(cgli_ctx *ctx, double *norms, int max_iters, int *iters);
/* Initial guess of each step's inner iteration.  0: Q^(n+1,0) = Q^n, as
 * main.cpp:364-386 leaves it; 1: second-order extrapolation
 * 3Q^n - 3Q^(n-1) + Q^(n-2) (2Q^n - Q^(n-1) for the first step after
 * cgli_set_state has one level of history); 2: extrapolation plus the
 * learned correction of the network given to cgli_set_learned_guess
 * (extrapolation while fewer than two levels of history exist, and in any
 * cell where the network's output is not finite). */
int cgli_set_predictor(cgli_ctx *ctx, int mode);

/* Bound of the device-side waits of the LU-SGS wavefront passes on other
 * tiles (the reference has none: its OpenMP barriers wait without limit): a
 * tile waiting for its neighbour's products polls at most `polls` times
 * (default CGLI_WAIT_LIMIT_DEFAULT, well over a second), then records a
 * timeout; from then on no wait of the pass waits again, the pass runs to
 * its end computing values that are discarded, the update leaves U_
 * unchanged, the call returns CGLI_ETIMEOUT and the next call runs normally.
 * 0 makes those waits give up at once (for tests of the timeout path). */
#define CGLI_WAIT_LIMIT_DEFAULT 4194304
int cgli_set_wait_limit(cgli_ctx *ctx, int polls);
/* The (i, j) column tile of the wavefront passes this library was built
 * with for CGLI_FP64 or CGLI_MIXED passes (no counterpart in the reference,
 * which sweeps whole hyperplanes): each pass takes
 * Nz + ti + tj - 2 + ti (ceil(Nx/ti) - 1) + tj (ceil(Ny/tj) - 1) dependent
 * steps.  Host only. */
int cgli_sweep_tile_shape(int precision, int *ti, int *tj);

/* ---- learned initial guess (no counterpart in the reference).  A 3-D
 * convolutional network, 15 -> 32 -> 32 -> 32 -> 32 -> 5 channels, 3x3x3
 * kernels, GELU after the first four layers, periodic in x and z, zero
 * padded at the walls, BF16 weights and activations with FP32 accumulation
 * on the tensor cores.  Input, from Q = U*J of Q^n, Q^(n-1), Q^(n-2):
 * channel v (Q^n_v - mean_v) / std_v, channel 5 + v (Q^n - Q^(n-1))_v / d1_v,
 * channel 10 + v (Q^n - 2Q^(n-1) + Q^(n-2))_v / d2_v; output: the correction
 * (Q^(n+1) - (3Q^n - 3Q^(n-1) + Q^(n-2)))_v / oscale_v.
 * Parameters: a flat float array, per layer W[27][cout][cin] (tap
 * t = (dx*3 + dy)*3 + dz for offsets dx-1, dy-1, dz-1) then b[cout].
 * The grid must have Ny a multiple of 4 and Nz a multiple of 32. */
typedef struct cgli_cnn cgli_cnn;
long long cgli_cnn_param_count(void);
int cgli_cnn_create(int nx, int ny, int nz, cgli_cnn **out);
int cgli_cnn_destroy(cgli_cnn *cnn);
const char *cgli_cnn_last_error(void);
int cgli_cnn_set_params(cgli_cnn *cnn, const float *theta);   /* also resets Adam */
int cgli_cnn_get_params(cgli_cnn *cnn, float *theta);
/* mean, std: of the level; d1, d2: RMS of its first and second time
 * differences; oscale: of the correction (all positive) */
int cgli_cnn_set_scales(cgli_cnn *cnn, const double mean[5], const double std[5], const double d1[5],
                        const double d2[5], const double oscale[5]);
/* x0: [15][Nx][Ny][Nz] already normalised; out: [5][Nx][Ny][Nz] */
int cgli_cnn_forward_host(cgli_cnn *cnn, const float *x0, float *out);
/* mean squared error against target [5][Nx][Ny][Nz] and its gradient with
 * respect to the flat parameters (the training step without the update) */
int cgli_cnn_loss_grad_host(cgli_cnn *cnn, const float *x0, const float *target, float *loss, float *grad);
/* training data: a ring of `count` stored time levels (physical Q, float) on
 * the device; pair p = (levels p, p+1, p+2 as history, level p+3 as target) */
int cgli_cnn_reserve_levels(cgli_cnn *cnn, int count);
long long cgli_cnn_levels(const cgli_cnn *cnn);
int cgli_cnn_push_level_host(cgli_cnn *cnn, const float *q);  /* [5][Nx][Ny][Nz] */
int cgli_cnn_push_level(cgli_cnn *cnn, cgli_ctx *ctx);         /* the context's Q^n (after cgli_step) */
int cgli_cnn_pair_loss(cgli_cnn *cnn, long long pair, float *loss);
/* `steps` Adam steps (learning rate lr) on pairs drawn uniformly (seeded)
 * from [first_pair, first_pair + npairs); mean training loss */
int cgli_cnn_train(cgli_cnn *cnn, int steps, float lr, unsigned long long seed, long long first_pair,
                   long long npairs, float *mean_loss);
/* device time (ms, mean over reps) of the network's inference on the
 * context's current levels: input packing and the five layers */
int cgli_cnn_time_inference(cgli_cnn *cnn, cgli_ctx *ctx, int reps, float *ms);
/* use the network for predictor mode 2 (null detaches it) */
int cgli_set_learned_guess(cgli_ctx *ctx, cgli_cnn *cnn);

/* ---- running statistics (replaces the accumulation of Statistic.cpp:120-160).
 * Each call adds, for every interior (i, j), the sums over k of U, V, W, T,
 * UU, VV, WW, TT, UV, UT, VT of the current U_ (call after each cgli_step),
 * and records the instantaneous U and T of the cell at reference index
 * k = 150 (Statistic.cpp:155-158; zero where Nz < 149);
 * cgli_statistics_get copies the [CGLI_NSTATS][Nx][Ny] values
 * (quantity-major, i then j: the 11 sums, then U and T at k = 150) and the
 * number of accumulated calls; the reference's means are the sums divided
 * by calls * Nz (Statistic.cpp:162-190). */
#define CGLI_NSTATS 13
int cgli_statistics_accumulate(cgli_ctx *ctx);
int cgli_statistics_get(cgli_ctx *ctx, double *sums, long long *samples);
int cgli_statistics_reset(cgli_ctx *ctx);

/* ---- high-order filter sensor (replaces Filter(myid, Roe_criterion, E_high,
 * E_low, U1_..U5_, Y_point, EpX, EpY, EpZ, J), Filter.cpp:12-1720, prototype
 * main.h:948-974).  Reads U_ as stored (ghost planes included, like the
 * reference: call cgli_halo_x and the boundary conditions first for fresh
 * ghosts), J and "Y_point" (set with cgli_set_array first, otherwise
 * CGLI_ESTATE); writes "EpX"/"EpY"/"EpZ" (read them with cgli_get_array)
 * over the reference's face ranges, E_high where the h / 2h velocity-energy
 * ratio of the face is >= roe_criterion, else E_low.  The two x-end faces of
 * EpX read the periodic image of the slab (the reference leaves those planes
 * of its E arrays unset on an interior rank).  The filter buffers (18 fields)
 * are allocated on first use. */
int cgli_filter(cgli_ctx *ctx, double roe_criterion, double e_high, double e_low);

/* Device timing on the context stream: record CUDA event `slot` (0..7) and
 * read the milliseconds between two recorded slots (synchronises on b). */
int cgli_event_record(cgli_ctx *ctx, int slot);
int cgli_event_elapsed(cgli_ctx *ctx, int a, int b, float *ms);
/* Device time of the wavefront passes (LU-SGS) of every inner iteration run
 * through cgli_inner_iteration / cgli_step since the last reset, from two
 * events recorded around them inside the iteration graph: total ms and the
 * number of passes (4 per inner iteration); reset != 0 clears the totals. */
int cgli_sweep_time(cgli_ctx *ctx, double *ms, long long *passes, int reset);

/* Stage timing of one inner iteration of the fast path, each stage launched
 * on its own between CUDA events on the context stream, `reps` times; writes
 * the mean milliseconds of CGLI_NSTAGES stages to ms[] in the order
 * halo+boundaries, x flux, y flux, z flux, viscous terms, residual assembly,
 * forward sweep pass, backward sweep pass (the last one with the update).
 * Leaves the state advanced by `reps` inner iterations. */
#define CGLI_NSTAGES 8
int cgli_profile_stages(cgli_ctx *ctx, int reps, double *ms);

/* No counterpart in the reference.  The primitive update and the five
 * residual norms of one inner iteration (the arithmetic of
 * Dual_time_stepping.cpp:1702-1782 and of the context path) on caller-owned
 * device arrays, for callers that cannot allocate device memory when they
 * need this step: a host code whose memory pool owns every device buffer, a
 * time loop that must not pay the synchronisation an allocation can imply,
 * or a process that has committed the whole GPU to its own arrays.  Nothing
 * is allocated: the per-row partial sums live in one static device array of
 * CGLI_NOALLOC_MAX_ROWS x 5 doubles (5 MiB, held by every GPU that loads the
 * library until the process exits).
 *   U_[5]  Q^(n+1,m)/J, updated in place; J; NR[5] the final sweep increments,
 *          all device pointers in the reference layout of an Nx x Ny x Nz slab;
 *   er[5]  host output, sqrt(sum of squared increments) / (Nx Ny Nz) for
 *          rho, u, v, w, p/rho; stream: a cudaStream_t or NULL.
 * Rejects Nx*Ny > CGLI_NOALLOC_MAX_ROWS with CGLI_EINVAL.  Every call looks up
 * the array's device address on the current device (cudaGetSymbolAddress,
 * which allocates nothing), so the address stays right after the device's
 * context is reset.  Each device holds its own copy of the array; on one
 * device all calls share it and it keeps the last call's contents (each call
 * overwrites the rows it reads, nothing has to start at zero), so calls that
 * overlap on the same device -- concurrent streams or host threads -- race
 * and must be serialised by the caller; calls on different devices do not.
 * Returns after the norms are on the host. */
#define CGLI_NOALLOC_MAX_ROWS 131072
int cgli_update_norms_noalloc(int nx, int ny, int nz, double *const U_[5], const double *J,
                              const double *const NR[5], double er[5], void *stream);

/* Hyperplane.cpp:18-80: cells of the interior slab listed by plane
 * m = i+j+k (m = 7 .. Nx+Ny+Nz+4), then i, j, k; Nijk[2*m] = running end
 * index, Nijk[2*m+1] = count; ijk[3*n..3*n+2] for n = 1..Nx*Ny*Nz.  Host
 * only, O(N) (the reference's brute force is O(N * planes)).  nijk_len and
 * ijk_len are the element counts of the buffers. */
int cgli_hyperplane(int nx, int ny, int nz, int *Nijk, long nijk_len, int *ijk, long ijk_len);

#ifdef __cplusplus
}
#endif
#endif
