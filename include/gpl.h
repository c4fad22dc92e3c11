/*
 * gpl_b200 — the C ABI of the B200 global-placement engine.
 *
 * The engine is a drop-in for the `global_placement` command of vyges-gpl. Every entry point
 * below names the reference interface it replaces (file:line within the vyges-gpl crate).
 * Plain C types only: the caller owns the arrays it passes; the library copies what it keeps.
 * All coordinates are database units (DBU).
 */
#ifndef GPL_B200_H
#define GPL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* How a run ended: `Stop` (src/log.rs:18-21) and the CLI's exit codes (src/main.rs:503-509).
 * GPL_DEVICE_FAULT has no reference counterpart: a CUDA error, reported with its text in
 * `reason`; the process is never aborted. */
#define GPL_PLACED 0
#define GPL_ERROR 2
#define GPL_REFUSED 3
#define GPL_DEVICE_FAULT (-1)

/* Outcome of a placed run (src/run.rs:35-48). */
#define GPL_OUTCOME_PLACED 0
#define GPL_OUTCOME_INITIALLY_PLACED 1

/* Instance flags (`DbInst`, src/placer_base.rs:52-75). */
#define GPL_INST_CORE_AUTO_PLACEABLE 1u
#define GPL_INST_BLOCK 2u
#define GPL_INST_FIXED 4u
#define GPL_INST_PLACED 8u
#define GPL_INST_HAS_HALO 16u

/* Orientations (`orient_point`, src/initial_place.rs:68-79). */
#define GPL_R0 0
#define GPL_R90 1
#define GPL_R180 2
#define GPL_R270 3
#define GPL_MY 4
#define GPL_MYR90 5
#define GPL_MX 6
#define GPL_MXR90 7

/* Port flags (`Port`, src/placer_base.rs:102-107). */
#define GPL_BTERM_PLACED 1u
#define GPL_BTERM_FIXED 2u

/*
 * The design as the placer reads it: `Design` (src/placer_base.rs:185-206) flattened into
 * arrays. Rectangles are 4 int32 (lx, ly, ux, uy). CSR starts have one more entry than their
 * owners. Name arrays may be NULL (names are then generated: "i<k>", "n<k>", "p<k>", "g<k>").
 */
typedef struct gpl_design {
  int32_t dbu;
  int32_t die[4];
  int32_t core[4];
  int32_t n_rows;
  const int32_t *row_box;      /* 4 per row */
  const uint8_t *row_pad;      /* the row's site class is PAD */
  const int32_t *row_site;     /* 2 per row: site width, height */
  int32_t n_insts;
  const int32_t *inst_box;     /* 4 per instance: getBBox() */
  const uint32_t *inst_flags;  /* GPL_INST_* */
  const int32_t *inst_group;   /* index into the groups, -1 for none */
  const int32_t *inst_halo;    /* 4 per instance, read when GPL_INST_HAS_HALO; may be NULL */
  const int32_t *inst_signal_pins;
  const uint8_t *inst_orient;  /* GPL_R0 .. GPL_MXR90 */
  const int32_t *inst_master;  /* 2 per instance: master width, height */
  const char *const *inst_name;
  const char *const *inst_master_name;
  int32_t n_nets;
  const uint8_t *net_signal;   /* SIGNAL or CLOCK */
  const int64_t *net_iterm_start;
  const int32_t *iterm_inst;
  const int32_t *iterm_shape;  /* 4 per terminal, master coordinates */
  const uint8_t *iterm_has_shape;
  const int32_t *iterm_order;  /* position among its instance's terminals */
  const int64_t *net_bterm_start;
  const int32_t *bterm_box;    /* 4 per port */
  const uint8_t *bterm_flags;  /* GPL_BTERM_* */
  const char *const *net_name;
  const char *const *bterm_name;
  int32_t n_groups;
  const char *const *group_name;
  const uint8_t *group_visual_debug;
  const int32_t *group_region; /* -1 for none */
  int32_t n_regions;
  const int32_t *region_bound_start;
  const int32_t *region_bounds; /* 4 per boundary */
  const int32_t *region_group_start;
  const int32_t *region_groups;
  int32_t n_blockages;
  const int32_t *blockage_box;
  const int32_t *blockage_inst;       /* -1 for none */
  const uint8_t *blockage_inst_fixed;
  const float *blockage_max_density;
} gpl_design_t;

/*
 * The routing services routability-driven placement calls: `trait Router`
 * (src/route_base.rs:90-126), the RUDY part. Each returns 0 on success. `net_term_boxes` is
 * called twice per pass: with boxes == NULL to get the count, then to fill `cap` entries.
 */
typedef struct gpl_router {
  void *user;
  /* Router::write_locations (src/route_base.rs:92): n triples (design instance, x, y). */
  int (*write_locations)(void *user, int64_t n, const int32_t *locations);
  /* Router::rudy_inputs (src/route_base.rs:99): die, grid, tile size, up to 32 pitches. */
  int (*rudy_inputs)(void *user, int32_t die[4], int32_t *x_grids, int32_t *y_grids,
                     int32_t *tile_size, int32_t *n_pitches, int32_t pitches[32]);
  /* Router::capacity_reduction (src/route_base.rs:102): x-major (capacity, reduction) bytes. */
  int (*capacity_reduction)(void *user, uint8_t *cap_red, int64_t n_tiles);
  /* Router::net_term_boxes (src/route_base.rs:125): design net index and box per net. */
  int64_t (*net_term_boxes)(void *user, int32_t *net_index, int32_t *boxes, int64_t cap);
} gpl_router_t;

/*
 * What one run returns: the JSON report's fields (src/main.rs:249-262, :362-371) and the
 * written placement (`placed_locations`, src/nesterov.rs:4099-4110). Library-owned memory,
 * released by gpl_result_free.
 */
typedef struct gpl_result {
  int32_t status;        /* GPL_PLACED / GPL_ERROR / GPL_REFUSED / GPL_DEVICE_FAULT */
  int32_t outcome;       /* GPL_OUTCOME_* when placed */
  char code[16];         /* "GPL-0307" on GPL_ERROR */
  char *reason;          /* refusal or device-fault text */
  char *lines;           /* the run's lines, each ended by '\n' */
  char *trace;           /* raw-value probe lines, each ended by '\n' */
  int64_t insts, nets, pins;
  int32_t iterations;    /* final Nesterov iteration, -1 when Nesterov did not run */
  int32_t n_bases;
  int32_t *bases;        /* 4 per base: group (-1 top level), placed, fixed, dummies */
  int64_t n_locations;
  int32_t *locations;    /* 3 per instance: design instance, lower-left x, lower-left y */
  int64_t final_hpwl;    /* the placer's HPWL over its pins at the end */
  float final_overflow;  /* average unscaled overflow at the end */
  int64_t trials;        /* back-tracking trials run */
  double seconds_initial_place;
  double seconds_nesterov;
  int64_t h2d_bytes;     /* host-to-device bytes the run copied */
  int64_t d2h_bytes;     /* device-to-host bytes the run copied */
  int64_t launches;      /* kernel launches the run made */
} gpl_result_t;

typedef struct gpl_ctx gpl_ctx;

/* One context binds one CUDA device and its own stream. Calls on one context are not
 * reentrant; contexts are independent. Returns NULL when the device cannot be used.
 * A finished command's host copies (the design, the placer's arrays: about 1 GB at 1M cells)
 * are freed by a thread of the context after the command has written its result, so the call
 * returns without waiting for them; at most one such thread runs (a command that ends while
 * the previous one's copies are still being freed waits for that first), and gpl_destroy
 * waits for it. Nothing the caller passed or received is touched by it. */
gpl_ctx *gpl_create(int device);
void gpl_destroy(gpl_ctx *ctx);

/* Engine options with no reference counterpart (the reference runs on one thread):
 *   "poisson" = "mixed" (split-BF16 tcgen05 DCT GEMMs, the default) | "fp32" (SIMT GEMMs) |
 *               "fp64" (the same transforms in double throughout: the precision yardstick)
 *   "trace"   = "0" | "1" (probe lines, as the reference's `Log.trace`)
 *   "reorder" = "1" (the default) | "0": the device's cell order sorted again by position when
 *               the cells have moved apart (no result depends on the order but the double sums'
 *               last bits), or kept as uploaded
 *   "packed"  = "auto" (the default: on with more than one region) | "1" | "0": each Nesterov
 *               phase (scatter, bin finalize, FP32 density solve, gradient update) of every
 *               region in one launch, or one launch a region; the results are the same bit
 *               for bit
 * Returns 0, or -1 for an unknown name or value. */
int gpl_set_option(gpl_ctx *ctx, const char *name, const char *value);

/* The `global_placement` proc: `run::global_placement` (src/run.rs:115). `argv` holds the
 * command's arguments (src/run.rs:16-30 keys and flags); `router` may be NULL (routability
 * is then refused, as src/run.rs:192). Returns out->status. */
int gpl_global_placement(gpl_ctx *ctx, const gpl_design_t *design, int argc,
                         const char *const *argv, const gpl_router_t *router,
                         gpl_result_t *out);
void gpl_result_free(gpl_result_t *out);

/* The same command with its Nesterov loop stepped by the caller: `open` is `run::global_placement`
 * up to the loop (construction, `do_initial_place`, `init_nesterov_place`, `init_nesterov_loop`:
 * src/run.rs:115-159, src/nesterov.rs:4123-4127); `iterate` runs up to n iterations of
 * `resume_nesterov_place`'s loop (src/nesterov.rs:4478-4575) and sets *done when the loop has
 * ended; `close` finishes it and writes the result as gpl_global_placement does. A stop in
 * `open` or `iterate` is reported by `close`. */
typedef struct gpl_session gpl_session;
gpl_session *gpl_session_open(gpl_ctx *ctx, const gpl_design_t *design, int argc,
                              const char *const *argv, const gpl_router_t *router);
int gpl_session_iterate(gpl_session *s, int n, int *done);
/* "poisson" = "mixed" | "fp32" | "fp64" (solvers rebuilt, the field recomputed); "profile" = "0" | "1"
 * (per-phase device time from CUDA events); "overlap" = "1" | "0" (the WA beside the density
 * solve or after it); "reorder" and "packed" as gpl_set_option's. No reference counterpart. */
int gpl_session_set_option(gpl_session *s, const char *name, const char *value);
/* Per-phase device milliseconds and launch counts since "profile" was set: scatter, bin
 * finalize, density solve, WA, gradients, HPWL. Returns the number of phases written. */
int gpl_session_profile(gpl_session *s, double *ms, int64_t *launches, int cap);
/* Kernel launches, host-to-device and device-to-host bytes since the session opened, the
 * Nesterov cells (instances and fillers) on the device, the back-tracking trials run
 * (`do_back_tracking`'s passes, src/nesterov.rs:2776-2808) and the times the engine sorted its
 * device cells again (the "reorder" option) since the session opened (6 int64). */
void gpl_session_counters(gpl_session *s, int64_t out[6]);
/* The Nesterov regions on the device: for each (up to cap) its bin grid (nx, ny), its cells
 * (instances and fillers) and its density solver's form (0 FP32, 1 split-BF16 tensor cores,
 * 2 FP64), 4 int32 a region. Returns the region count. */
int gpl_session_regions(gpl_session *s, int32_t *out, int cap);
/* The engine's autotuner so far, as text: for each tuned launch group (the small nets' WA
 * form, each region's scatter form) the form in use and its candidates' median times in
 * microseconds. Writes at most cap bytes (NUL included) to buf; returns the text's length. */
int gpl_session_tuning(gpl_session *s, char *buf, int cap);
/* The session's CUDA stream (cudaStream_t), for timing with events on it. */
void *gpl_session_stream(gpl_session *s);
int gpl_session_close(gpl_session *s, gpl_result_t *out);
/* Drops a session where it stands: no loop to the end, no result. */
void gpl_session_discard(gpl_session *s);

/* A stand-in for the database's router (src/db_router.rs:260-368): a uniform tile grid over
 * the die, the given pitches, every tile with `capacity` and no reduction, and each net's
 * terminal box from its pin shapes at the written locations. No reference counterpart. */
gpl_router_t *gpl_synthetic_router_create(const gpl_design_t *design, int32_t tile_size,
                                          int32_t n_pitches, const int32_t *pitches,
                                          uint8_t capacity);
void gpl_synthetic_router_destroy(gpl_router_t *router);

/* ---- per-kernel entry points, for per-kernel parity and benchmarks ----
 * Device pointers on the caller's stream (cudaStream_t passed as void*). Each returns 0, or a
 * CUDA error code. None has a reference entry point of its own; each names the function whose
 * result it computes. */

/* The bin-density scatter `update_bins_gcell_density_area` (src/nesterov.rs:2218-2250):
 * cells' density boxes (integer centre cx, cy; half sizes hx, hy; density scale; kind 0 std
 * cell, 1 macro, 2 filler) over a grid of nx * ny bins whose lower-left is (grid_lx, grid_ly),
 * edges bx[0..nx], by[0..ny], bin sizes size_x, size_y. Writes the int64 accumulators
 * inst[nx*ny] and filler[nx*ny] (x-major: index x*ny + y), zeroed first. */
int gpl_kernel_density_scatter(int64_t n_cells, const int32_t *cx, const int32_t *cy,
                               const int32_t *hx, const int32_t *hy, const float *scale,
                               const uint8_t *kind, int32_t nx, int32_t ny, int32_t grid_lx,
                               int32_t grid_ly, const int32_t *bx, const int32_t *by,
                               double size_x, double size_y, float target_density,
                               int64_t *inst, int64_t *filler, void *stream);

/* The Nesterov step `nesterov_update_coordinates` (src/nesterov.rs:2718-2746, with
 * `inside_x/y` :2188-2213) up to the field, as one trial runs it: per cell (float pairs x, y)
 *   next     = clamp(cur_slp + step * cur_slp_sum),
 *   next_slp = clamp(next' + coeff * (next' - cur))  (next' the unclamped next),
 * each clamped so the density box (half sizes hx, hy: 2 hx wide, as `set_density_size` leaves
 * it) stays inside the grid [grid_lx, bx[nx]] x [grid_ly, by[ny]]; a locked cell (locked may be
 * NULL) keeps cur and cur_slp. Then the density centre at next_slp, truncated to integers
 * (`update_gcell_density_center_location`, :2268-2276), into centre (2 per cell), and the bin
 * scatter of those boxes as gpl_kernel_density_scatter writes it into inst and filler (zeroed
 * first). Float pairs and centre must be 8-byte aligned. */
int gpl_kernel_nesterov_step(int64_t n_cells, const float *cur_slp, const float *cur_slp_sum,
                             const float *cur, const int32_t *hx, const int32_t *hy,
                             const float *scale, const uint8_t *kind, const uint8_t *locked,
                             int32_t nx, int32_t ny, int32_t grid_lx, int32_t grid_ly,
                             const int32_t *bx, const int32_t *by, double size_x, double size_y,
                             float target_density, float step, float coeff, float *next,
                             float *next_slp, int32_t *centre, int64_t *inst, int64_t *filler,
                             void *stream);

/* `update_gradients` (src/nesterov.rs:2455-2507) with the step length's distances
 * (`distance`, :319-330): per cell, the WA force summed over its pins in its own order
 * (`wl_gradient`, :2418-2430; pin_force holds each pin's force times its net's weight, cell-major:
 * the cell's pins at cell_pin_start[i] .. cell_pin_start[i+1]), the density force over its bins,
 * x outer, y inner (`density_gradient`, :2434-2449; centre 2 per cell, fields x-major), and
 *   sum = (wl + penalty * density) / max(pins + penalty * area, 1)
 * into sum (2 per cell). sums (host, 4 doubles) receives sum |wl|, sum |density|,
 * sum |a1 - b1|^2 (a1 and b1 both NULL: 0) and sum |sum - b2|^2 (b2 NULL: 0) over every cell's
 * x and y, each in double. Float pairs and centre must be 8-byte aligned. */
int gpl_kernel_gradients(int64_t n_cells, const int32_t *centre, const int32_t *hx,
                         const int32_t *hy, const float *scale, const float *area,
                         const int64_t *cell_pin_start, const float *pin_force, int32_t nx,
                         int32_t ny, int32_t grid_lx, int32_t grid_ly, const int32_t *bx,
                         const int32_t *by, double size_x, double size_y, const float *field_x,
                         const float *field_y, float penalty, float *sum, const float *a1,
                         const float *b1, const float *b2, double *sums, void *stream);

/* `get_hpwl` (src/nesterov.rs:2297-2304): the sum over nets (pins net-major, net_start[n_nets+1])
 * of each net's pin-box half perimeter, int64, into *hpwl (host). fused = 1 takes it from the WA
 * kernels, which add it up beside the forces as each trial reads it back; 0 from the HPWL
 * kernels an iteration runs without a WA pass. */
int gpl_kernel_hpwl(int64_t n_nets, const int64_t *net_start, const int32_t *pin_xy,
                    int32_t fused, int64_t *hpwl, void *stream);

/* `Fft::solve` (src/nesterov.rs:412-444) without the potential: density[nx*ny] (x-major) to
 * field_x, field_y (device pointers). mode 0 = FP32 SIMT GEMMs, 1 = split-BF16 tcgen05 GEMMs,
 * 2 = the FP32 form's transforms in double (fields rounded to float once).
 * wx[nx], wy[ny] are the wavenumbers (host pointers). Builds its basis matrices and workspace
 * per call, so it allocates. */
int gpl_kernel_poisson(int32_t nx, int32_t ny, const float *wx, const float *wy,
                       const float *density, float *field_x, float *field_y, int mode,
                       void *stream);

/* `update_wirelength_force_wa` + `wl_gradient_pin` (src/nesterov.rs:2325-2414): per net (pins
 * net-major, net_start[n_nets+1]), per pin its position pin_xy[2*p], pin_xy[2*p+1];
 * coefficients coef_x, coef_y; writes each pin's force (gmin - gmax) scaled by its net's weight
 * (net_weight may be NULL: 1) into grad[2*n_pins]. */
int gpl_kernel_wa(int64_t n_nets, const int64_t *net_start, const int32_t *pin_xy,
                  const float *net_weight, float coef_x, float coef_y, float *grad, void *stream);

/* `Csr::from_triplets` (src/bicgstab.rs:501-541, the initial placement's collapse) on device
 * arrays: n rows, nt triplets (row, col, val) in their order; duplicates summed in that order,
 * each row's columns ascending. Writes row_start[n+1], and *nnz (host) entries into cols and
 * vals (device buffers of at least nt entries). Rows of any length: a warp, a block or a
 * thread per row by length, the same result from each. */
int gpl_kernel_csr_from_triplets(int64_t n, int64_t nt, const int32_t *rows, const int32_t *cols,
                                 const float *vals, int64_t *row_start, int32_t *out_cols,
                                 float *out_vals, int64_t *nnz, void *stream);

/* `Csr::mul` (src/bicgstab.rs:72-82): y = A x on a CSR matrix (device pointers), each row's
 * products summed in column order, then 0 + 1 * sum, as the solver forms them. form picks the
 * kernel: GPL_SPMV_ROWS (a thread per row), GPL_SPMV_TILED (a block's products staged in
 * shared memory) or GPL_SPMV_SLICED (a thread per row over a copy of the matrix in slices of
 * 32 rows stored column-major, built by the call, which then synchronizes the stream); all
 * give the same y, bit for bit. */
#define GPL_SPMV_ROWS 0
#define GPL_SPMV_TILED 1
#define GPL_SPMV_SLICED 2
int gpl_kernel_spmv(int64_t n, const int64_t *row_start, const int32_t *cols, const float *vals,
                    const float *x, float *y, int32_t form, void *stream);

/* The initial placement's solver `bicgstab` (src/bicgstab.rs:615-669) on a CSR matrix (device
 * pointers) with FP64 inner products; x is the start point and the result. Writes iterations
 * and error (host pointers). Allocates its scratch vectors per call. */
int gpl_kernel_bicgstab(int64_t n, const int64_t *row_start, const int32_t *cols,
                        const float *vals, const float *rhs, float *x, int32_t max_iters,
                        int32_t *iterations, float *error, void *stream);

/* gpl_kernel_bicgstab without any device allocation. This entry point has no counterpart in the
 * reference. It is for callers that cannot call cudaMalloc: code held to a device-memory pool
 * sized in advance, which a library must not bypass; hosts that forbid a plug-in library to
 * allocate device memory on its own; and code that shares the GPU with latency-critical
 * streams, where cudaMalloc and cudaFree may wait for the whole device. Its scratch is one fixed device array of this
 * library, so it serves systems of at most GPL_BICGSTAB_NOALLOC_MAX_ROWS rows (about 3.7 MB of
 * scratch); a larger n returns GPL_NOALLOC_TOO_LARGE and touches nothing, a negative n
 * cudaErrorInvalidValue. The driver reserves the array on a device when it loads the library's
 * device code there: under CUDA's default lazy module loading, at the first use of the
 * library's kernels on that device (possibly inside this entry point's first call); with
 * CUDA_MODULE_LOADING=EAGER, when the context is made. It is held until the process exits. The
 * first call on a device also looks up the array's device address there (cudaGetSymbolAddress,
 * with that device current): a caller that budgets device memory or captures streams makes one
 * call on each device before doing so. The address is kept for the process, so after
 * cudaDeviceReset on a device this entry point must not be called on that device again. Every call on a device
 * shares the one array, so calls that overlap on the GPU (other streams, other threads) race:
 * serialise them. Arguments and results as gpl_kernel_bicgstab's. */
#define GPL_BICGSTAB_NOALLOC_MAX_ROWS 131072
#define GPL_NOALLOC_TOO_LARGE (-2)
int gpl_kernel_bicgstab_noalloc(int64_t n, const int64_t *row_start, const int32_t *cols,
                                const float *vals, const float *rhs, float *x,
                                int32_t max_iters, int32_t *iterations, float *error,
                                void *stream);

/* RUDY `Rudy::calculate` (src/route_base.rs:191-253): net boxes (4 per net) into a tile
 * demand map (x-major, cnt_x * cnt_y) over tiles of `tile_size` from the die's lower-left,
 * the last column and row stretched to `die_ux`, `die_uy`. */
int gpl_kernel_rudy(int64_t n_nets, const int32_t *boxes, int32_t die_lx, int32_t die_ly,
                    int32_t die_ux, int32_t die_uy, int32_t cnt_x, int32_t cnt_y,
                    int32_t tile_size, int32_t wire_width, float *demand, void *stream);

/* The density solve of gpl_kernel_poisson in double precision throughout (basis matrices,
 * products, spectral step): the yardstick the FP32 and split-BF16 forms' errors are reported
 * against. Fields as double, x-major. No reference counterpart in this precision: it is the
 * exact transform the reference's float Ooura transforms approximate. */
int gpl_kernel_poisson_fp64(int32_t nx, int32_t ny, const float *wx, const float *wy,
                            const float *density, double *field_x, double *field_y,
                            void *stream);

/* ---- the objectives and their adjoints (double precision, device pointers) ----
 * The reference takes only the gradients (forces) of its two objectives: the WA wirelength's
 * in `update_wirelength_force_wa` + `wl_gradient_pin` (src/nesterov.rs:2325-2430) and the
 * electrostatic energy's in `density_gradient` (:2434-2449) over `Fft::solve` (:412-444).
 * These entry points give the values and their exact derivatives, for gradient checks by
 * finite differences and for callers that differentiate through the objective.
 *
 * WA: W = sum_n w_n sum_{axis} (sum x e^{c x} / sum e^{c x} - sum x e^{-c x} / sum e^{-c x})
 * over each net's pins (pin_xy[2*p], pin_xy[2*p+1]), exact exponentials, coefficient c per
 * axis. The backward writes seed * dW/d(pin x, y) into grad[2*n_pins]. */
int gpl_fn_wa_forward(int64_t n_nets, const int64_t *net_start, const double *pin_xy,
                      const float *net_weight, double coef_x, double coef_y, double *value,
                      void *stream);
int gpl_fn_wa_backward(int64_t n_nets, const int64_t *net_start, const double *pin_xy,
                       const float *net_weight, double coef_x, double coef_y, double seed,
                       double *grad, void *stream);
/* Electrostatic energy E = 1/2 rho^T G rho over nx * ny uniform bins of bin_w x bin_h from
 * (grid_lx, grid_ly): rho the cells' overlap areas (centre cell_xy[2*i..], half sizes
 * half[2*i..]) times their density scales, G the reference's DCT Poisson solve. The backward
 * writes seed * dE/d(cell x, y) into grad[2*n_cells]. */
int gpl_fn_density_forward(int64_t n_cells, const double *cell_xy, const double *half,
                           const double *scale, int32_t nx, int32_t ny, double grid_lx,
                           double grid_ly, double bin_w, double bin_h, double *energy,
                           void *stream);
int gpl_fn_density_backward(int64_t n_cells, const double *cell_xy, const double *half,
                            const double *scale, int32_t nx, int32_t ny, double grid_lx,
                            double grid_ly, double bin_w, double bin_h, double seed,
                            double *grad, void *stream);
/* The same objective with its grid planned once (the DCT bases on the device, the solve's
 * buffers), for many evaluations: eval writes the energy (when energy is not NULL) and
 * seed * dE/d(cell x, y) into grad (when grad is not NULL) for the cells given. create
 * returns NULL for an empty grid or a failed allocation. */
typedef struct gpl_fn_density gpl_fn_density;
gpl_fn_density *gpl_fn_density_create(int32_t nx, int32_t ny, double grid_lx, double grid_ly,
                                      double bin_w, double bin_h, void *stream);
int gpl_fn_density_eval(gpl_fn_density *f, int64_t n_cells, const double *cell_xy,
                        const double *half, const double *scale, double *energy, double seed,
                        double *grad);
void gpl_fn_density_destroy(gpl_fn_density *f);

#ifdef __cplusplus
}
#endif

#endif /* GPL_B200_H */
