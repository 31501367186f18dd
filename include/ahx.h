/* ahx.h — C ABI of the B200 live solver: the coupled D3Q19 flow + D3Q7 heat lattice-Boltzmann step of the
 * ashburn-heat-twin live mode, on CUDA (sm_100a).
 *
 * The host keeps the domain and parameter math (js/live/domain.js and the parameter code of js/live/solver.js in the
 * reference) and hands this library the same byte images the reference's WebGPU backend receives:
 *   - the parameter block, 64 + 16*nz bytes (kernel.js:36-50, written by solver.js:225-242);
 *   - the per-column records, NXY x vec4<u32> = (kt, ktop, cd f32 bits, q f32 bits) (solver.js:359-376);
 *   - the ktop plane, NXY x u32 (solver.js:338).
 * Populations are exchanged in the reference's layout, f32 [q][cell] with cell = (k*ny + j)*nx + i, j = 0 at the
 * south edge (kernel.js:17), whatever the internal storage format.
 *
 * Conventions: every call returns an ahx_status (0 = ok). On failure ahx_last_error() returns a readable message for
 * the calling thread. A handle owns all device memory it uses; host buffers are always the caller's and are copied
 * in or out before the call returns (or, for ahx_read_submit, before ahx_read_wait returns). Calls on one handle are
 * serialised by an internal mutex. Device work is queued on the handle's CUDA stream and returns at once unless the
 * call says otherwise. A CUDA error on the handle's context makes the handle "lost": later calls return
 * AHX_EDEVICE (the reference's device-lost state, solver.js:139,219-222). No call aborts or traps.
 */
#ifndef AHX_H
#define AHX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AHX_OK = 0,
  AHX_EINVAL = 1,      /* bad argument or size */
  AHX_ENOMEM = 2,      /* device or pinned-host allocation failed (solver.js:142-156 out-of-memory scope) */
  AHX_EDESTROYED = 3,  /* handle already destroyed (solver.js:220 "live solver: destroyed") */
  AHX_EDEVICE = 4,     /* CUDA error: the handle is lost (solver.js:221) */
  AHX_ETIMEOUT = 5,    /* a bounded wait expired; the work is still queued */
  AHX_ENONFINITE = 6,  /* a check found NaN/Inf in the state */
  AHX_EBUSY = 7        /* no free read slot (more than AHX_MAX_READS reads in flight) */
} ahx_status;

/* storage of the populations (arithmetic is f32, f64 for AHX_FP64). The 16-bit formats store (f - w) * scale for the
 * flow populations; AHX_FP16_G32 / AHX_BF16_G32 store f in 16 bits and the temperature populations g in f32, which
 * keeps the heat budget (a per-step source increment can be far below half an ulp of a 16-bit g). AHX_FP16_SR is
 * the AHX_FP16 format whose step rounds stochastically (a dither keyed on the cell and a per-handle step counter,
 * deterministic for a given history): unbiased rounding instead of round-to-nearest's persistent bias. */
typedef enum {
  AHX_FP32 = 0,
  AHX_FP16 = 1,
  AHX_BF16 = 2,
  AHX_FP64 = 3,
  AHX_FP16_G32 = 4,
  AHX_BF16_G32 = 5,
  AHX_FP16_SR = 6
} ahx_precision;

/* step output modes (kernel.js:427-428; solver.js:551-558 stepOut / stepAcc) */
typedef enum { AHX_MODE_NONE = 0, AHX_MODE_OUT = 1, AHX_MODE_ACC = 2 } ahx_mode;

/* arithmetic variant of the fused step: EXACT evaluates every expression in the reference's order with IEEE-rounded
 * f32 operations and no contraction (bit-identical to the CPU restatement); FAST lets the compiler contract into FMA. */
typedef enum { AHX_ARITH_EXACT = 0, AHX_ARITH_FAST = 1 } ahx_arith;

#define AHX_MAX_READS 8

typedef struct ahx_handle ahx_handle;

typedef struct {
  int32_t nx, ny, nz;        /* grid (reference: dom.nx, ny, nz) */
  int32_t precision;         /* ahx_precision of the stored populations */
  int32_t device_ordinal;    /* CUDA device; -1 = current */
  int32_t arith;             /* ahx_arith */
} ahx_dims;

typedef struct {
  int32_t nx, ny, nz, px;    /* px: internal x pitch in elements */
  int32_t precision, arith, parity, device_ordinal;
  int64_t steps;             /* steps run on this handle since creation */
  uint64_t state_bytes;      /* bytes of both population buffers */
  uint64_t bytes_per_cell;   /* algorithmic bytes moved per fluid cell update (read + write of f and g) */
  char device_name[64];
} ahx_info_out;

/* diagnostics over all fluid cells of the current state (kernel.js:580-633 genStatsWGSL, solver.js:559-575):
 * per-cell f32 values summed in FP64 */
typedef struct {
  double sum_theta;          /* sum of theta (K) */
  double sum_ke;             /* sum of 0.5|j|^2/rho (lattice units) */
  double sum_rho_dev;        /* sum of rho - 1 */
  double count;              /* fluid cells with finite rho and theta */
  float theta_max;           /* max(theta, 0) */
  float umax;                /* max |j|/rho (lattice units) */
  uint32_t non_finite;       /* cells with non-finite rho or theta */
  uint32_t pad;
} ahx_stats_out;

/* Per-step FP64 budget record, accumulated inside the fused step when enabled (no counterpart in the reference,
 * which computes the heat budget offline from time-mean fields, tools/live/validate_live.py:226-240). Lateral-face
 * sums use the post-stream moments of the face cells: theta*u (K lattice-velocity) and u (lattice velocity). */
typedef struct {
  double theta_sum;          /* sum of pre-collision theta over fluid cells */
  double src_sum;            /* sum of the per-column source S (K/step) injected this step */
  double face_theta_u[4];    /* sum over face cells of theta*u_n: west (ux), east (ux), south (uy), north (uy) */
  double face_u[4];          /* sum over face cells of u_n, same faces */
  double cells;              /* fluid cells updated */
  double pad[5];
} ahx_budget_out;

/* --- lifetime ------------------------------------------------------------------------------------------------ */

/* createLiveSolver's device part (solver.js:137-196 _init: buffers; pipelines are compiled ahead of time here).
 * Allocates both population buffers, column and ktop planes and the read pool. */
ahx_status ahx_create(const ahx_dims* dims, ahx_handle** out);

/* destroy() (solver.js:485-493): idempotent for a valid handle; releases everything. */
ahx_status ahx_destroy(ahx_handle* h);

/* thread-local message of the last failure on this thread */
const char* ahx_last_error(void);

ahx_status ahx_get_info(ahx_handle* h, ahx_info_out* out);

/* --- host images (solver.js:225-242, 323-376) ------------------------------------------------------------------ */

/* the parameter block: bytes == 64 + 16*nz (kernel.js:36) */
ahx_status ahx_set_params(ahx_handle* h, const void* params, size_t bytes);

/* NXY records of 4 x u32 (kt, ktop, cd bits, q bits) */
ahx_status ahx_set_columns(ahx_handle* h, const uint32_t* colv);

/* the ktop plane; when old_ktop is not NULL, cells that turned from solid to fluid (k in [ktop, min(old_ktop, nz)))
 * get rest equilibrium and theta = 0 in the current state (solver.js:336-349 + kernel.js:557-575 genReinitWGSL) */
ahx_status ahx_set_ktop(ahx_handle* h, const uint32_t* ktop, const uint32_t* old_ktop);

/* --- state (solver.js:288-293, 380-398) ------------------------------------------------------------------------ */

/* f -> equilibrium with the inflow profile at the local height above terrain in both buffers (kernel.js:524-553
 * genInitWGSL); theta kept; the stochastic-rounding step counter restarts (AHX_FP16_SR) */
ahx_status ahx_init_flow(ahx_handle* h);

/* g -> 0 in both buffers (solver.js:383,394 clearBuffer) */
ahx_status ahx_clear_heat(ahx_handle* h);

/* set the ping-pong parity (resetFlow sets 0, solver.js:396) */
ahx_status ahx_set_parity(ahx_handle* h, int parity);

/* --- stepping (solver.js:401-427) ------------------------------------------------------------------------------- */

/* queue n fused steps (kernel.js:395-431). mode AHX_MODE_OUT writes (theta, ux, uy, uz) on the last step,
 * AHX_MODE_ACC accumulates it on every step. Returns at once. */
ahx_status ahx_step(ahx_handle* h, int n, int mode);

/* queue n steps bracketed by two CUDA events recorded on the handle's own stream, wait for them (bounded by
 * timeout_ms, < 0 = no limit) and return the device time between the events in *ms */
ahx_status ahx_time_steps(ahx_handle* h, int n, int mode, int timeout_ms, float* ms);

/* wait for all queued work; timeout_ms < 0 waits without limit. AHX_ETIMEOUT leaves the work queued. */
ahx_status ahx_sync(ahx_handle* h, int timeout_ms);

/* a fence after the work queued so far: ahx_fence returns a ticket, ahx_fence_query reports 1 when it passed */
ahx_status ahx_fence(ahx_handle* h, uint64_t* ticket);
ahx_status ahx_fence_query(ahx_handle* h, uint64_t ticket, int* done);

/* --- read-back (solver.js:439-471; kernel.js:435-520) ----------------------------------------------------------- */

/* queue the near-surface and volume extraction of the current state behind the queued steps and start the copy to
 * pinned staging on a second stream; stepping may continue meanwhile. conv = dx/dt (f32), volscale = 255/volMax
 * (f32), nzv levels of u8 volume. Returns a ticket for ahx_read_wait. */
ahx_status ahx_read_submit(ahx_handle* h, float conv, float volscale, int nzv, int want_vol, int want_wind,
                           uint64_t* ticket);

/* wait (bounded) for a submitted read and copy it out: surf/u/v NXY f32 north-up (u, v may be NULL), vol
 * nzv*NXY u8 (may be NULL), theta_max the unclamped max theta over the fluid cells of those levels. */
ahx_status ahx_read_wait(ahx_handle* h, uint64_t ticket, int timeout_ms, float* surf, float* u, float* v,
                         uint8_t* vol, float* theta_max);

/* --- validation hooks (solver.js:496-578 _dbg) ------------------------------------------------------------------ */

ahx_status ahx_read_state(ahx_handle* h, float* f, float* g);          /* 19N + 7N f32, reference layout */
ahx_status ahx_write_state(ahx_handle* h, const float* f, const float* g); /* either may be NULL */
ahx_status ahx_read_state_f64(ahx_handle* h, double* f, double* g);    /* FP64 handles only */
ahx_status ahx_write_state_f64(ahx_handle* h, const double* f, const double* g);
ahx_status ahx_read_dbg(ahx_handle* h, float* dbg4);                   /* 4N f32 (theta, ux, uy, uz) per cell */
ahx_status ahx_clear_dbg(ahx_handle* h);
ahx_status ahx_stats(ahx_handle* h, ahx_stats_out* out);               /* synchronous */

/* --- budgets ---------------------------------------------------------------------------------------------------- */

/* enable (1) / disable (0) the per-step FP64 budget accumulation fused into the step; while enabled each step adds
 * into a device record, read (and optionally reset) with ahx_budget_read (synchronous). */
ahx_status ahx_budget_enable(ahx_handle* h, int on);
ahx_status ahx_budget_read(ahx_handle* h, ahx_budget_out* out, int reset);

/* Time accumulators, no counterpart in the reference (it takes its time means offline from the +32 B/cell
 * accumulate mode, tools/live/validate_live.py:226-255). While enabled, every step adds, in FP64: per column at its
 * first fluid cell (theta, ux, uy) in lattice units, solver orientation [j][i] (j = 0 south); per lateral-face cell
 * (theta, u_n): west then east faces as [k][j], then south then north faces as [k][i]. Enabling allocates and zeroes
 * them; ahx_accum_read copies the sums (surf3: 3 * nx * ny doubles; faces: 2 * (2 ny nz + 2 nx nz) doubles; either may
 * be NULL) and the number of steps accumulated, optionally resetting both (synchronous). */
ahx_status ahx_accum_enable(ahx_handle* h, int on);
ahx_status ahx_accum_read(ahx_handle* h, double* surf3, double* faces, int64_t* steps, int reset);

/* --- tuning ----------------------------------------------------------------------------------------------------- */

/* launch shape of the fused step: block_y = threads per block in y (x is one warp) plus 100 x the register-budget
 * variant (0: compiler's choice; 4, 5, 6 or 8: 128-thread blocks, that many resident per SM, only with block_y 4), plus
 * 2000 for paired levels (two interior levels per thread on packed f32x2 arithmetic; FMA build, f32 arithmetic; the
 * results are bit-identical to unpaired), plus 10000 for an L2 prefetch of the next level's source rows (FMA build;
 * a hint that changes no result); or, for the TMA-staged kernel, 1000 + 100 x stages + rows (rows 4 with 2-4 stages,
 * rows 8 with 2-3 stages; 4- and 8-byte storages); or, for the TMA-staged paired step of the 16-bit storages (FP16,
 * BF16, FP16 with stochastic rounding; FMA build; whole domains), 2000 + 1000 + 100 x stages + rows (rows 4 or 8 with
 * 2-4 / 2-3 stages; bit-identical to the plain paired step); zslab = z-slab depth in levels (rounded up to even for
 * the staged paired step); 0 = keep */
ahx_status ahx_set_launch(ahx_handle* h, int block_y, int zslab);
/* time candidate launch shapes on scratch copies of the state and keep the fastest; the state is not advanced;
 * *best_block_y uses the encoding of ahx_set_launch */
ahx_status ahx_autotune(ahx_handle* h, int steps_per_trial, int* best_block_y, int* best_zslab, float* best_ms);

/* --- diagnostics without allocation ---------------------------------------------------------------------------- */

/* No counterpart in the reference. The ahx_stats diagnostics (theta, kinetic energy, rho - 1 and fluid-cell sums in
 * FP64, max theta, max |j|/rho, non-finite count) over a state the caller owns, for callers that cannot allocate
 * device memory when they need them: an engine that has given all device memory to its own pool, code that must not
 * block on a driver allocation.
 * f (19N) and g (7N) are f32 device arrays in the reference layout, ktop is the NXY device plane, out is an
 * ahx_stats_out in device memory; the two kernels run on `stream` (a cudaStream_t; NULL = the legacy default stream)
 * and the call returns once they are queued. Nothing is allocated: the per-block partial sums go to one fixed
 * 1 MiB scratch array inside the library (held by every GPU that loads it until the process exits), so grids above
 * 134,217,728 cells are rejected with AHX_EINVAL. The first call on a device (and the first after the device's
 * context changed, e.g. after cudaDeviceReset) resolves that array's address: make that call before any stream
 * capture. Calls share the array: two calls that overlap on the GPU race on it. The sums are
 * reduced in a fixed order, so repeated calls on the same state return identical records. */
ahx_status ahx_stats_noalloc(int nx, int ny, int nz, const float* f, const float* g, const uint32_t* ktop,
                             ahx_stats_out* out, void* stream);

/* --- y-slab decomposition of one domain ----------------------------------------------------------------------- */

/* No counterpart in the reference (one domain per device). A handle can hold rows [jg0, jg0 + ny) of a domain nyg
 * rows tall and update only its local rows [jlo, jhi); the other local rows are ghost copies of the neighbouring
 * slabs' boundary rows, refreshed after every step by copying packed rows between slabs (ahx_row_pack on one,
 * ahx_row_unpack on the other; device buffers, ordered on each handle's stream; over NCCL between GPUs). Lateral
 * faces and the outflow sponge follow the global rows, so the stepped rows are bit-identical to the undivided
 * domain's. Slabs use the plain kernels (no staged kernel, no batches); stats count only the updated rows. */
ahx_status ahx_set_slab(ahx_handle* h, int jg0, int nyg, int jlo, int jhi);
/* bytes of a packed row: [19][nz][nx] f elements, padded to 16 bytes, then [7][nz][nx] g elements; the buffers given
 * to ahx_row_pack / ahx_row_unpack must be 16-byte aligned */
ahx_status ahx_row_bytes(ahx_handle* h, size_t* bytes);
ahx_status ahx_row_pack(ahx_handle* h, int j, void* dst_device);
ahx_status ahx_row_unpack(ahx_handle* h, int j, const void* src_device);
/* The halo of a boundary: of local row j, only the populations that cross to the neighbour, c_y = dir (+1: the 5 flow
 * and 1 temperature populations moving north, which the north slab's first row pulls from its ghost row; -1: those
 * moving south), 6 of the 26 planes. Packed as [5][nz][nx] f elements, padded to 16 bytes, then [nz][nx] g elements
 * (ahx_halo_bytes); buffers 16-byte aligned. ahx_halo_pack reads the current state (next = 0) or the state the step in
 * progress writes (next = 1, between ahx_step_rows calls of one step); ahx_halo_unpack writes the current state. */
ahx_status ahx_halo_bytes(ahx_handle* h, size_t* bytes);
ahx_status ahx_halo_pack(ahx_handle* h, int j, int dir, int next, void* dst_device);
ahx_status ahx_halo_unpack(ahx_handle* h, int j, int dir, const void* src_device);
/* One step in parts: update only local rows [j0, j1) (within the rows the handle updates) from the current state into
 * the next one; the call with advance = 1 completes the step (the state read by later calls flips). A slab steps its
 * boundary rows first, packs their halos (next = 1) for the neighbours, and then its interior rows, so the halo
 * transfer overlaps the interior update. The parts of a step are bit-identical to one whole step. Not for
 * AHX_FP16_SR storage or with budgets or accumulators enabled (AHX_EINVAL). */
ahx_status ahx_step_rows(ahx_handle* h, int j0, int j1, int advance);

/* --- batched stepping ----------------------------------------------------------------------------------------- */

/* No counterpart in the reference, which steps one domain per device (solver.js:401-427). A batch groups handles of
 * one device, precision and arithmetic (grids may differ) so that each step of all of them is ONE persistent launch
 * (a member's result is bit-identical to stepping it alone), replayed two steps at a time from a CUDA graph. Members
 * stay usable on their own (parameters, columns, reads, solo steps): the batch's launches are ordered after the work
 * already queued on each member's stream and before anything queued there later. A member cannot be destroyed while
 * it belongs to a batch (AHX_EINVAL), and batched steps do not accumulate budgets or time sums (members with either
 * enabled are rejected). Tiles are 32 x 4 columns x 8 levels, handed to the persistent blocks from a device counter in list order;
 * the register-budget variant is the members' tuned one when they agree, else 4. ahx_batch_set_launch overrides
 * both. */
typedef struct ahx_batch ahx_batch;

typedef struct {
  int members, tiles, grid, minb, use_graph, zslab_max, pairs, pad;
  int64_t cells;   /* sum of nx*ny*nz over the members */
} ahx_batch_info_out;

ahx_status ahx_batch_create(ahx_handle* const* members, int count, ahx_batch** out);
/* replace the member list (count >= 0; same device, precision and arithmetic); stream-ordered after the batch's
 * earlier steps, without synchronising or allocating unless the batch outgrows its tables; the captured graph stays
 * valid. Members that leave are released (they may then be destroyed: their streams already wait for the batched
 * steps that used them). */
ahx_status ahx_batch_set_members(ahx_batch* b, ahx_handle* const* members, int count);
/* n steps of every member, asynchronous; each member's step count and parity advance as with ahx_step */
ahx_status ahx_batch_step(ahx_batch* b, int n);
/* n batched steps timed with CUDA events on the batch stream; waits at most timeout_ms (< 0: no bound) */
ahx_status ahx_batch_time_steps(ahx_batch* b, int n, int timeout_ms, float* ms);
ahx_status ahx_batch_sync(ahx_batch* b, int timeout_ms);
/* launch set-up: register-budget variant 4 / 5 / 6 (0 = keep); tile depth zslab in levels for every member (clipped
 * to its nz; 0 = keep; -1 = whole columns when that leaves at least 4 tiles per persistent block, else each member's
 * own z-slab); use_graph: 1 = steps replay the captured graph of the persistent launch, 0 = one persistent launch per
 * step, 2 = steps replay a graph of each member's own solo step kernel (its own launch shape, e.g. from
 * ahx_autotune) on parallel branches, which the device runs concurrently (minb, zslab and pairs then do not apply);
 * paired levels on packed f32x2 arithmetic (1 on, 0 off, -1 keep; FMA build, f32 arithmetic only) */
ahx_status ahx_batch_set_launch(ahx_batch* b, int minb, int zslab, int use_graph, int pairs);
ahx_status ahx_batch_get_info(ahx_batch* b, ahx_batch_info_out* out);
ahx_status ahx_batch_destroy(ahx_batch* b);   /* idempotent; members are released */

/* --- domain builder on the GPU --------------------------------------------------------------------------------- */

/* The host's domain and column images (js/live/domain.js loadStatic10 :32-69, aggregate :89-118, rasterizeCampuses
 * :124-160, buildDomain :166-190; the column record of solver.js:359-376) built by kernels instead: the 10 m static
 * planes are uploaded and decoded once (the dem's row-wise int16 first differences summed per row), each grid spacing
 * is block-aggregated once, and each request's campuses, building rule and column records take three small launches.
 * Every result is bit-identical to the host restatement (double precision in the reference's operation order). */
typedef struct ahx_static ahx_static;

/* raw: the decompressed static10 payload; offsets: byte offsets of the planes dem (low-byte plane, then high-byte
 * plane, nrows * ncols each), lc (u8), frac25 (u8), hmean (u16 little-endian), dca4 (u8), as static10.json lists them */
ahx_status ahx_static_create(int device_ordinal, int nrows, int ncols, const uint8_t* raw, size_t raw_bytes,
                             const size_t* offsets, ahx_static** out);
/* integer sums of the decoded planes, for the reference's checksums: dem (cm), lc, frac25, hmean (cm), dca4 */
ahx_status ahx_static_checksums(ahx_static* s, int64_t* sums);
ahx_status ahx_static_destroy(ahx_static* s);   /* idempotent */

typedef struct {
  double dx;                 /* grid spacing (m): a multiple of 10 that divides the box */
  double heightM;            /* domain height (m) */
  double extra_height;       /* minimum building height where a campus adds roof area (m; the reference uses 14) */
  int32_t nz_min;            /* lower bound of nz (0: none) */
  int32_t ncampus;           /* campuses, in list order */
  const double* campus_mw;   /* heat load of each campus (MW) */
  const int32_t* hall_count; /* halls of each campus */
  const double* halls;       /* sum of hall_count entries of [x0, z0, x1, z1] (scene metres) */
  double* campus_flux;       /* out: W per m^2 of each campus's total hall roof */
  double flux_existing;      /* W per m^2 of operational data-center roof */
  double kq;                 /* dt / (rho cp dx^3): K per step per W in one cell */
  const double* cd_table;    /* 256 drag coefficients by land-cover class: (kappa / ln(0.5 dx / z0))^2 */
} ahx_domain_spec;

typedef struct {
  int32_t nx, ny, nz, ktop_max;
  double zbase;              /* floor(min dem) - dx (m) */
  int64_t nb_cells;          /* building cells (sum of nb) */
} ahx_domain_out;

/* build one request's geometry: colv (4 * NXY u32: kt, ktop, cd f32 bits, q f32 bits) and ktop (NXY) in solver
 * orientation (row 0 south), and the north-up campus heat (W) and new roof area (m^2) per cell; any output may be
 * NULL. Synchronous. */
ahx_status ahx_domain_build(ahx_static* s, const ahx_domain_spec* spec, ahx_domain_out* out, uint32_t* colv,
                            uint32_t* ktop, double* heat_w, double* new_area);

/* --- serving: continuous batching behind the C ABI -------------------------------------------------------------- */

/* No counterpart in the reference: the live page serves one scenario at a time (js/live.js:69-86 steps it and reads
 * it back in a loop). A server runs many scenario solves ("requests") on one device. The host builds each request's
 * byte images exactly as for ahx_set_params / ahx_set_columns / ahx_set_ktop (the scenario's setMet,
 * setExistingFlux and setNewCampuses, solver.js:225-376) and submits them with a step count and the read-back
 * settings of ahx_read_submit. A scheduler thread inside the library admits requests in arrival order while the
 * resident cells stay under max_cells and the slots' device memory under the HBM budget; it configures a solver slot
 * (recycled from finished requests of the same grid, or created) as resetFlow would (equilibrium flow, theta 0, parity
 * 0), steps every active request together in chunks of at most `chunk` steps with the batched launch (ahx_batch_*:
 * each slot's own tuned step kernel on parallel graph branches, or one persistent launch), never past any request's
 * step count, changes the member list between chunks (requests join and leave while others run: continuous
 * batching), and answers a finished request with the read-back of its final state. Each answer is bit-identical to
 * the same scenario stepped alone on a fresh handle. Host buffers are copied at submit and copied out at poll; the
 * server owns all device memory. All calls are thread-safe. */
typedef struct ahx_server ahx_server;

typedef struct {
  int32_t device_ordinal;    /* CUDA device; -1 = current */
  int32_t precision, arith;  /* ahx_precision / ahx_arith of every slot */
  int32_t chunk;             /* steps per batched chunk (<= 0: 256) */
  int64_t max_cells;         /* resident-cell budget (<= 0: 24,000,000) */
  uint64_t hbm_budget_bytes; /* device memory the slots may hold (0: 80 % of the memory free at creation) */
  int32_t batch_mode;        /* 0: each slot's own step kernel on parallel graph branches; 1: one persistent launch */
  int32_t tune;              /* 1: tune the launch shape on the first slot of each grid (ahx_autotune), reuse it */
  int32_t depth;             /* chunks queued ahead of the scheduler (<= 0: 2) */
  int32_t pad;
} ahx_server_config;

typedef struct {
  int32_t nx, ny, nz;        /* grid of the scenario */
  int32_t steps;             /* steps to run (>= 0) */
  const void* params;        /* parameter block, params_bytes == 64 + 16 nz */
  size_t params_bytes;
  const uint32_t* colv;      /* 4 * nx * ny column records */
  const uint32_t* ktop;      /* nx * ny ktop plane */
  float conv, volscale;      /* read-back scaling, as ahx_read_submit */
  int32_t nzv, want_vol, want_wind;
  int32_t pad;
  uint64_t user_tag;         /* returned in ahx_server_result */
} ahx_request;

typedef struct {
  uint64_t ticket, user_tag;
  int32_t nx, ny, nz, nzv, steps, status;    /* status: AHX_OK, or the error that ended the request */
  double submitted_s, admitted_s, done_s;    /* seconds since the server was created */
  float theta_max;                            /* unclamped max theta of the read-back levels */
  int32_t want_vol, want_wind, pad;
} ahx_server_result;

typedef struct {
  int64_t submitted, admitted, completed, queued, active;
  int64_t cell_updates;      /* nx * ny * nz * steps summed over the chunks launched */
  int64_t chunks, batch_steps, slots, idle_slots, evictions, resident_cells;
  uint64_t slot_bytes, hbm_budget_bytes;
  double elapsed_s;          /* since creation */
} ahx_server_stats_out;

ahx_status ahx_server_create(const ahx_server_config* cfg, ahx_server** out);
/* copy the request in and queue it; returns its ticket at once */
ahx_status ahx_server_submit(ahx_server* s, const ahx_request* req, uint64_t* ticket);
/* wait up to timeout_ms (< 0: no bound) for the request; when it is done, fill *info and copy its read-back out
 * (surf, u, v: nx * ny f32 north-up, u / v only with want_wind, vol: nzv * nx * ny u8 with want_vol; any may be NULL)
 * and release the ticket. AHX_ETIMEOUT: not finished yet (the ticket stays valid). Returns the request's status. */
ahx_status ahx_server_poll(ahx_server* s, uint64_t ticket, int timeout_ms, ahx_server_result* info, float* surf,
                           float* u, float* v, uint8_t* vol);
ahx_status ahx_server_stats(ahx_server* s, ahx_server_stats_out* out);
/* stop the scheduler (requests not answered yet are dropped), release every slot and the batch; idempotent */
ahx_status ahx_server_destroy(ahx_server* s);

#ifdef __cplusplus
}
#endif

#endif /* AHX_H */
