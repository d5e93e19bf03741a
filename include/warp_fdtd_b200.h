/*
 * warp_fdtd_b200 — C ABI of the B200 (sm_100a) uniform-grid FDTD library.
 *
 * Every entry point takes raw device pointers, sizes and a cudaStream_t passed
 * as void* (NULL = legacy default stream), launches asynchronously on that
 * stream and returns FDTD_OK (0) or a negative status; nothing is allocated or
 * freed and no ownership is transferred.  fdtd_last_error() returns a message
 * for the last failure on the calling thread.
 *
 * Layout (warp_fdtd/kernels.py:25): a field is (3, n) float32, n = nx*ny*nz,
 * flat index i = (x*ny + y)*nz + z with z fastest.  A 2-D argument is passed
 * with its column count ("*_cols") so that arrays of other widths (such as the
 * reference tests' (3, 1) placeholders) are addressed as the reference does.
 *
 * Two groups of entry points:
 *  1. Kernel-level replacements of the reference's Warp kernels, same
 *     arguments in the same order and the same in-place semantics.  Each cites
 *     the kernel it replaces.
 *  2. The B200 forward path the Solver uses: one fused E+H step over
 *     ping-pong buffers plus float64 multi-frequency detector recorders.
 */
#ifndef WARP_FDTD_B200_H
#define WARP_FDTD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_OK 0
#define FDTD_ERR_ARG (-1)   /* invalid size, pointer or option */
#define FDTD_ERR_CUDA (-2)  /* a CUDA launch or runtime call failed */

/* Message for the last non-zero status returned on this thread. */
const char *fdtd_last_error(void);

/* Library ABI version (major*100 + minor). */
int fdtd_version(void);

/* ---------------------------------------------------------------------------
 * 1. Kernel-level replacements
 * ------------------------------------------------------------------------ */

/* Replaces kernels.py:77-148 update_e / update_h / update_e_packed /
 * update_h_packed (`make_update(electric, packed)`), launched over n cells.
 * f (3, fg_cols) is updated in place from g; psi (6, psi_cols) holds f's CPML
 * state; coeff is (3, clen, 3) float (a, b, 1/kappa) or, with packed != 0,
 * (3, clen, 4) with the plane rank of solver.py:16-29 pack_coefficients;
 * source (3, source_cols) and waves (3, waves_cols) inject the plane source
 * at x == source_x (source_x < 0 disables it); step is the device step
 * counter; when electric == 0 and step >= save_h_from the old H is copied to
 * hprev (3, hprev_cols).  periodic != 0 wraps neighbours (kernels.py:19-22). */
int fdtd_update(int electric, int packed, float *f, const float *g, long long fg_cols,
                const float *inv_eps, float *psi, long long psi_cols, const float *coeff,
                int clen, const float *source, long long source_cols, const float *waves,
                long long waves_cols, const int *step, float *hprev, long long hprev_cols,
                int save_h_from, int nx, int ny, int nz, int source_x, float courant,
                int periodic, void *stream);

/* Replaces kernels.py:151-153 `advance` (delta = +1) and adjoint.py:226-228
 * `retreat` (delta = -1): step[0] += delta on the device. */
int fdtd_advance(int *step, int delta, void *stream);

/* Replaces detectors.py:65-106 `record`, launched over count = sx*sy*sz
 * plane cells starting at (x0, y0, z0).  weights is (steps, 2) float32
 * (complex64 as re, im), indices (steps) int32, phasor (6, count, 2) float32,
 * flux (bins) float32, area (count) float32.  Fields e, h, prev are (3, cols).
 * Phasor cells accumulate exactly as the reference (float32); flux bins are
 * added with float32 atomics, as the reference does. */
int fdtd_record(const float *e, const float *h, const float *prev, long long cols,
                const int *step, const float *weights, const int *indices, float *phasor,
                float *flux, const float *area, int nx, int ny, int nz, int x0, int y0,
                int z0, int sx, int sy, int sz, int axis, int exact, int is_phasor,
                void *stream);

/* Replaces adjoint.py:17-43 `record_curl`: hist[step, c, j] = courant *
 * curl(H)_c over the design box (x0, y0, z0, sx, sy, sz); hist is
 * (steps, 3, sx*sy*sz). */
int fdtd_record_curl(const float *h, long long cols, float *hist, const int *step, int nx,
                     int ny, int nz, int x0, int y0, int z0, int sx, int sy, int sz,
                     float courant, void *stream);

/* Replaces adjoint.py:46-88 `prepare` (transpose of the field scaling and the
 * CPML recurrence).  q (3, n), eps (n), psi (6, n), coeff (3, clen, 3),
 * d (6, n). */
int fdtd_prepare(const float *q, const float *eps, float *psi, const float *coeff, int clen,
                 float *d, int nx, int ny, int nz, float courant, int electric,
                 void *stream);

/* Replaces adjoint.py:107-162 `gather` (q += D^T d; with from_h, the design
 * inner product grad[j] += sum_c hist[step, c, j] * q_c).  grad is float32
 * (grad_f64 == 0, as the reference) or float64 (grad_f64 != 0). */
int fdtd_gather(float *q, const float *d, const float *hist, void *grad, int grad_f64,
                const int *step, int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                int sy, int sz, int from_h, void *stream);

/* One half of the reverse step, prepare + gather fused (adjoint.py:46-88 and
 * 107-162, as sequenced by adjoint.py:388-414), bitwise the reference
 * sequence without the d buffer.  from_h = 1: q_dst = qE, q_src = qH,
 * magnetic scaling, H CPML state, neighbours at -1, and (with grad)
 * grad[j] += hist[hist_step[0]] . q over the design box in float64; from_h =
 * 0: q_dst = qH, q_src = the updated qE, electric scaling with eps, E CPML
 * state, neighbours at +1.  The CPML state ping-pongs: psi0 is read and psi1
 * written when step[0] is even, the other way round when odd (step is the
 * reverse step counter, decremented once per reverse step); both start at
 * zero.  coeff is the CPML table padded to (3, clen, 4) floats (a, b,
 * 1/kappa, unused), 16-byte aligned, clen >= max(nx, ny, nz); nx <= 65535
 * and ny * nz < 2^31. */
int fdtd_reverse_half(int from_h, float *q_dst, const float *q_src, const float *eps,
                      float *psi0, float *psi1, const float *coeff, int clen, const int *step,
                      const float *hist, double *grad, const int *hist_step, int nx, int ny,
                      int nz, float courant, int x0, int y0, int z0, int sx, int sy, int sz,
                      void *stream);

/* Replaces adjoint.py:181-223 `inject` (transpose of detector colocation):
 * source (6, count, 2) float32, weights (steps, 2); scattered with float32
 * atomics as the reference does. */
int fdtd_inject(float *qe, float *qh, const float *source, const float *weights,
                const int *step, int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                int sy, int sz, int old_h_only, void *stream);

/* fdtd_inject for up to FDTD_INJECT_PLANES_MAX planes in one launch (the
 * adjoint's mode planes of one half step), each with its own source
 * (6, sx*sy*sz, 2), weights (steps, 2) and extent.  The same scattered sums;
 * float32 atomics, so the summation order differs from separate launches. */
#define FDTD_INJECT_PLANES_MAX 8
typedef struct fdtd_inject_plane {
    const float *source;
    const float *weights;
    int x0, y0, z0, sx, sy, sz;
} fdtd_inject_plane;
int fdtd_inject_many(float *qe, float *qh, const fdtd_inject_plane *planes, int nplanes,
                     const int *step, int nx, int ny, int nz, int old_h_only, void *stream);

/* Replaces adjoint.py:472-490 `write_design`: eps[box] = plane[x, y] for all z
 * in the box; plane is (sx, sy) float32. */
int fdtd_write_design(const float *plane, float *eps, int nx, int ny, int nz, int x0,
                      int y0, int z0, int sx, int sy, int sz, void *stream);

/* Replaces material.py:12-25 `smooth`: out = clamp-extended 2-D correlation
 * of p (px, py) with weights (2r+1, 2r+1), r = radius (the reference uses 9). */
int fdtd_material_smooth(const float *p, const float *weights, int radius, float *out,
                         int px, int py, void *stream);

/* Replaces material.py:35-55 `subpixel` (+ `project` 28-32): out =
 * 1 / (eps_lo + contrast * projected(rho)); the reference's map has
 * eps_lo = 1 and contrast = 11.25. */
int fdtd_material_subpixel(const float *rho, float *out, int px, int py, float beta,
                           float eps_lo, float contrast, void *stream);

/* Reverse mode of fdtd_material_subpixel (the reference differentiates it with
 * a Warp Tape, material.py:93-102): rho_grad += d out/d rho ^T g. */
int fdtd_material_subpixel_adjoint(const float *rho, const float *g, float *rho_grad,
                                   int px, int py, float beta, float eps_lo,
                                   float contrast, void *stream);

/* Reverse mode of fdtd_material_smooth: p_grad += smooth^T g (clamp edges fold
 * their weight back onto the edge pixel). */
int fdtd_material_smooth_adjoint(const float *g, const float *weights, int radius,
                                 float *p_grad, int px, int py, void *stream);

/* record_curl for the fused path's ping-pong buffers (adjoint.py:17-43): with
 * t = step[0] the H read by step t's E update is H[t & 1] (rows of pitch
 * pitch_z); hist[hist_step[0], c, j] = courant * curl(H)_c over the design
 * box; hist is (rows, 3, sx*sy*sz). */
int fdtd_record_curl_pp(const float *H0, const float *H1, int pitch_z, const int *step,
                        const int *hist_step, float *hist, int nx, int ny, int nz, int x0,
                        int y0, int z0, int sx, int sy, int sz, float courant, void *stream);

/* The whole material map of material.py:58-91 in one call: scratch (px*py
 * floats, caller-owned) receives smooth(p), out receives subpixel(scratch). */
int fdtd_material_forward(const float *p, const float *weights, int radius, float *scratch,
                          float *out, int px, int py, float beta, float eps_lo,
                          float contrast, void *stream);

/* fdtd_material_forward without the scratch argument, for callers that may not
 * allocate device memory themselves: an embedding application that owns a
 * fixed memory budget and hands the library only its input and output
 * buffers, or a control loop where a cudaMalloc (which can synchronise the
 * device) is not acceptable.  This entry point has no counterpart in the
 * reference.  The smoothed density lives in a static device array built into
 * the library, FDTD_MATERIAL_NOALLOC_MAX floats (1,048,576 = 4 MiB, held on
 * every GPU that loads the library until the process exits); px * py above
 * that limit is rejected with FDTD_ERR_ARG.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device
 * current, so make that first call before any stream capture.  The address
 * is kept for the life of the process: do not use this entry point on a
 * device after cudaDeviceReset (or any teardown of its primary context) in
 * the same process.  Every call
 * shares the one array: calls whose work overlaps on the GPU (other streams,
 * other threads) race and must be serialised by the caller.  Nothing in the
 * array needs clearing between calls; each call overwrites the px * py
 * entries it uses.  Allocates nothing. */
#define FDTD_MATERIAL_NOALLOC_MAX (1 << 20)
int fdtd_material_forward_noalloc(const float *p, const float *weights, int radius,
                                  float *out, int px, int py, float beta, float eps_lo,
                                  float contrast, void *stream);

/* Its pullback (material.py:93-102): p_grad = (d out / d p)^T g, overwritten.
 * scratch holds 2*px*py floats (the smoothed density and its adjoint). */
int fdtd_material_backward(const float *p, const float *weights, int radius, const float *g,
                           float *scratch, float *p_grad, int px, int py, float beta,
                           float eps_lo, float contrast, void *stream);

/* ---------------------------------------------------------------------------
 * 2. B200 forward path
 * ------------------------------------------------------------------------ */

/* Arguments of one fused leapfrog step (E then H), the work of
 * solver.py:194-237's update_e + update_h launches.  Buffers ping-pong: with
 * t = step[0] and s = t & 1 the step reads E[s], H[s], psi_*[s] and writes
 * E[s^1], H[s^1], psi_*[s^1], so after the step H[s] still holds H(n-1/2)
 * (the reference's hprev).  It does not advance step[0].
 *
 * Rows may be padded: cell (x, y, z) of a field, of full-storage psi and of
 * inv_eps lives at (x*ny + y)*pitch_z + z, and of the uint8 material at
 * (x*ny + y)*material_pitch + z.  Padding cells must hold zeros (fields) and
 * are never written.  The TMA paths need pitch_z % 4 == 0, material_pitch % 16
 * == 0 and 16-byte aligned buffers; path 3 also needs pitch_z <= 248 and the
 * slab psi layout.  Path 0 picks 3, then 2, then the shared-memory path 1. */
/* CPML state layouts of fdtd_step_args.packed:
 *  FDTD_PSI_FULL   (6, psi_cols) indexed by cell (solver.py cpml_storage="full");
 *  FDTD_PSI_PACKED (6, psi_cols) indexed by the reference's plane-rank formula
 *                  (kernels.py:50-74, cpml_storage="packed");
 *  FDTD_PSI_SLAB   per field one buffer holding three slab blocks, rows padded
 *                  to pitch_z: X [2][psi_rx][ny][pitch_z], then
 *                  Y [2][psi_ry][nx][pitch_z], then Z [2][nx][ny][psi_rz]
 *                  (psi_rz a multiple of 4); the slot pair of each axis is
 *                  (2*axis, 2*axis+1) and ranks come from coeff[...][3].  The
 *                  Z block is contiguous in z-rank so the full-z TMA path can
 *                  stage it with the fields.  Slab ranks are this layout's
 *                  own: every cell of a z window of active cells, widened to
 *                  whole groups of 4 (V) cells, gets consecutive ranks, so the
 *                  4 cells of a group with any active cell hold ranks
 *                  rb .. rb+3 with rb % 4 == 0 and rb + 4 <= psi_rz; a block
 *                  that finds otherwise sets *error = 2 and writes nothing. */
#define FDTD_PSI_FULL 0
#define FDTD_PSI_PACKED 1
#define FDTD_PSI_SLAB 2

typedef struct fdtd_step_args {
    float *E[2];
    float *H[2];
    float *psi_e[2];           /* (6, psi_cols) each */
    float *psi_h[2];
    long long psi_cols;        /* layouts 0/1: columns of each (6, psi_cols) psi array */
    const float *coeff_e;      /* (3, clen, 4): a, b, 1/kappa, packed plane rank */
    const float *coeff_h;
    int clen;
    int packed;                /* psi layout, see FDTD_PSI_* */
    int psi_rx, psi_ry, psi_rz; /* slab layout: active positions per axis (max of E, H) */
    int material_kind;         /* 0: inv_eps per cell, 1: uint8 index into table */
    const float *inv_eps;      /* per cell float32, material_kind 0 */
    const uint8_t *material;   /* per cell uint8, material_kind 1 */
    const float *material_table; /* (material_count) inverse permittivities */
    int material_count;        /* <= 256 */
    const float *src_e;        /* (3, ny*nz) E profile (drives the H update) */
    const float *src_h;        /* (3, ny*nz) H profile (drives the E update) */
    const float *waves_e;      /* (3, waves_cols) */
    const float *waves_h;
    long long waves_cols;      /* steps with t >= waves_cols inject nothing */
    int source_x;              /* < 0: no source */
    float courant;
    const int *step;
    int nx, ny, nz;
    int pitch_z;               /* 0: nz */
    int material_pitch;        /* 0: nz */
    int tile_y, tile_z, chunk_x; /* launch shape; 0 picks defaults */
    int path;                  /* 0 auto, 1 shared-memory staging, 2 TMA pipeline (tiled z),
                                  3 TMA pipeline over full-z tiles (needs FDTD_PSI_SLAB) */
    int vector;                /* TMA path: z cells per thread (1, 2, 4); 0 picks */
    int stages;                /* TMA path: planes in the load ring (2..8); 0 picks */
    int *error;                /* optional device int, set to 1 if a bounded wait expires */
    const int *schedule;       /* path 3, optional: schedule_blocks int4 entries in device
                                  memory, one per block: (y tile index, first x plane,
                                  end x plane, 0); null keeps the tile x chunk_x grid.
                                  chunk_x must be >= the longest entry's planes */
    int schedule_blocks;
} fdtd_step_args;

int fdtd_step_fused(const fdtd_step_args *args, void *stream);

/* Batches: many grids advanced by one launch of the full-z step.
 * fdtd_batch_prepare builds every grid's tensor maps and parameters (each
 * args[i] as for fdtd_step_fused with the slab psi layout, tile_y and chunk_x
 * set and equal across the batch, as are the row pitch, z slab width,
 * material kind and stages; schedule ignored) into `workspace` (device
 * memory of fdtd_batch_workspace_bytes(count) bytes, 64-byte aligned,
 * written synchronously: call it outside stream capture) and fills *plan.
 * fdtd_step_batch then runs one step of every grid with `blocks` blocks,
 * block b taking the int4 schedule entry b = (grid, y tile, first plane, end
 * plane) in device memory; each grid's own step[0] selects its parity, and
 * fdtd_advance_many advances the counters (steps: device array of `count`
 * device pointers).  Grid parameters live in a device-wide table of 128
 * slots shared by all live batches: fdtd_batch_release frees a batch's.  No
 * reference counterpart. */
typedef struct fdtd_batch_plan {
    int count, smem_bytes, threads, material_kind, stages, vector, full_rows;
    int base, device;  /* the batch's parameter slots (at most 128 grids live per device) */
} fdtd_batch_plan;

long long fdtd_batch_workspace_bytes(int count);
int fdtd_batch_prepare(const fdtd_step_args *args, int count, void *workspace,
                       long long workspace_bytes, fdtd_batch_plan *plan);
int fdtd_step_batch(const fdtd_batch_plan *plan, const void *workspace, const int *schedule,
                    int blocks, void *stream);
int fdtd_advance_many(int *const *steps, int count, int delta, void *stream);
/* Free a prepared batch's parameter slots (the workspace is the caller's).
 * No fdtd_step_batch launch of the plan may still be pending on the device:
 * a later fdtd_batch_prepare can take the slots and rewrite them at once.
 * fdtd_step_batch must run with the plan's device current. */
int fdtd_batch_release(fdtd_batch_plan *plan);

/* Time-blocked fused step: one launch advances E and H by `depth` (1 or 2)
 * time steps, the work of depth x solver.py:194-237's update_e + update_h
 * launches (kernels.py:77-148), reading every plane of E(n), H(n-1/2) once
 * and writing E(n+depth), H(n+depth-1/2) once.  Arguments and buffer
 * convention as fdtd_step_fused with the slab CPML layout (path 3): with t =
 * step[0] and s = t & 1 it reads E[s], H[s], psi_*[s] and writes E[s^1],
 * H[s^1], psi_*[s^1] (the depth-step result), and does not advance step[0].
 * Bitwise equal to `depth` single steps.  No reference counterpart (the
 * reference launches one sweep per field and step).
 *
 * fdtd_step_block_prepare (synchronous: call it outside stream capture)
 * reads the z CPML coefficients, orders the groups of four z cells so that the
 * ones carrying z CPML run in warps of their own, picks the tile (args->tile_y
 * or, when 0, the tallest that fits) and fills *plan.  args->stages (2..4,
 * default 2) sizes shared memory.  fdtd_step_block launches
 * args->schedule_blocks blocks, block b running the schedule's int4 entries
 * (y tile, first plane, end plane, 0) b*segments .. b*segments+segments-1 in
 * order (extra->segments, default 1; a tile < 0 ends the block's list, and
 * args->chunk_x must be at least the longest entry), or one block per tile x
 * chunk_x planes without a schedule.  extra may be NULL at depth 1.
 * Depth 2 keeps the CPML state between its two steps in `extra->scratch`
 * (plan->scratch_block_bytes per block, 16-byte aligned, no initial contents)
 * and can write E(n+1) and H(n+1/2) of the cells inside up to
 * FDTD_SNAP_BOXES_MAX boxes (x0, x1, y0, y1, z0, z1, half-open; whole groups
 * of four z cells) to snap_e / snap_h ((3, nx*ny*pitch_z) each), so that
 * detectors can sample the intermediate step.  Blocks below
 * extra->interior_blocks run a build of the kernel without the x/y CPML
 * code (schedule them on the grid's CPML-free interior).  args->error, when
 * set, receives 1 (a bounded wait expired), 2 (z CPML ranks not in groups of
 * four), 3 (a schedule entry outside the grid or longer than chunk_x) or 4
 * (an interior block's segment touches x/y CPML); the fields are then not
 * valid. */
#define FDTD_BLOCK_GROUPS_MAX 64
#define FDTD_SNAP_BOXES_MAX 8
typedef struct fdtd_block_plan {
    int depth, tile_y, stages, rows, threads;
    int groups_plain, groups_slab;   /* groups of 4 z cells without / with z CPML */
    unsigned char group[FDTD_BLOCK_GROUPS_MAX];  /* plain groups, then slab groups */
    long long scratch_block_bytes;   /* depth 2: scratch bytes per block */
    int pair_blocks;                 /* 1: two blocks per SM (registers capped) */
    int device, blocks_per_sm, sms;
} fdtd_block_plan;

typedef struct fdtd_block_extra {
    float *scratch;
    long long scratch_bytes;
    float *snap_e, *snap_h;
    int segments;  /* schedule entries per block (default 1): block b runs entries
                      b*segments .. b*segments+segments-1 in order, tile < 0 ends the list */
    int nsnap;
    int snap_box[FDTD_SNAP_BOXES_MAX][6];
    int interior_blocks; /* blocks [0, interior_blocks) run a build without x/y CPML code:
                            their segments (rows and planes xa-depth-1 .. xb+depth) must
                            carry no x/y CPML state and 1/kappa == 1, else error 4 */
} fdtd_block_extra;

int fdtd_step_block_prepare(const fdtd_step_args *args, int depth, fdtd_block_plan *plan);
int fdtd_step_block(const fdtd_step_args *args, const fdtd_block_plan *plan,
                    const fdtd_block_extra *extra, void *stream);

/* Fill the full-z path's launch-shape defaults into *args (tile_y where 0;
 * chunk_x where 0 and no schedule is set), as fdtd_step_fused would pick
 * them.  No reference counterpart. */
int fdtd_step_defaults(fdtd_step_args *args);

/* Resident blocks per SM of the full-z path's kernel for these arguments
 * (after the defaults fdtd_step_fused would pick) and the device's SM count,
 * for sizing a schedule to whole waves.  No reference counterpart. */
int fdtd_step_occupancy(const fdtd_step_args *args, int *blocks_per_sm, int *sms);

/* Float64 running DFT at one detector plane for K frequencies (the phasor
 * branch of detectors.py:65-106 generalised), run after fdtd_step_fused and
 * before the step counter advances.  With t = step[0] and s = t & 1 the new
 * fields are E[s^1], H[s^1] and H(n-1/2) is H[s] (the reference's hprev); the
 * field rows have pitch `pitch_z`.  If t < nsteps and indices[t] >= 0,
 * phasor[k, c, i] (re, im) += w[k, t] * f_c for the six colocated
 * (exact != 0) or raw components f_c, the fp32 sample and weight promoted to
 * float64.  indices (nsteps) int32; weights (K, nsteps, 2) float32; phasor
 * (K, 6, count, 2) float64. */
int fdtd_record_phasor64(const float *E0, const float *E1, const float *H0, const float *H1,
                         const int *step, const int *indices, int nsteps,
                         const float *weights, int nfreq, double *phasor, int nx, int ny,
                         int nz, int pitch_z, int x0, int y0, int z0, int sx, int sy, int sz,
                         int exact, void *stream);

/* Volume phasor observer (volume.py:60-89, record_volume) with float64
 * accumulators.  With t = step[0] and the buffer convention of
 * fdtd_record_phasor64, if first <= t < nsteps every sampling point i
 * (positions (count, 3) float32, grid units: position / spacing from the
 * grid's lower corner) gets phasor[c, i] (re, im) += weights[t] * f_c, where
 * f_c is component c trilinearly interpolated (zero outside the grid) at the
 * point minus the component's Yee offset, and H is the mean of H(n+1/2) and
 * H(n-1/2).  weights (nsteps, 2) float32; phasor (6, count, 2) float64. */
int fdtd_record_volume(const float *E0, const float *E1, const float *H0, const float *H1,
                       const int *step, const float *positions, long long count,
                       const float *weights, int nsteps, int first, double *phasor, int nx,
                       int ny, int nz, int pitch_z, void *stream);

/* Flux branch of detectors.py:104-106 with float64 bins, same buffer
 * convention as fdtd_record_phasor64: if t < nsteps and 0 <= indices[t] <
 * nbins, flux[indices[t]] += sum over the plane of cross(E, H)[axis] * area
 * (fp32 products summed in float64). */
int fdtd_record_flux64(const float *E0, const float *E1, const float *H0, const float *H1,
                       const int *step, const int *indices, int nsteps, const float *area,
                       double *flux, int nbins, int nx, int ny, int nz, int pitch_z, int x0,
                       int y0, int z0, int sx, int sy, int sz, int axis, int exact,
                       void *stream);

/* Batched form of fdtd_record_phasor64 for CUDA-graph step loops: each step
 * writes the six colocated (or raw) float32 samples of the plane into slot
 * t % T of `stage` ((T, 6, count) float32, count = sx*sy*sz), skipping steps
 * with t >= nsteps or indices[t] < 0; fdtd_dft_fold then adds the staged
 * steps to the float64 phasors.  Same buffer convention as
 * fdtd_record_phasor64. */
int fdtd_record_stage(const float *E0, const float *E1, const float *H0, const float *H1,
                      const int *step, const int *indices, int nsteps, float *stage, int T,
                      int nx, int ny, int nz, int pitch_z, int x0, int y0, int z0, int sx,
                      int sy, int sz, int exact, void *stream);

/* fdtd_record_stage for up to FDTD_STAGE_PLANES_MAX planes in one launch
 * (each plane with its own schedule, staging buffer and extent).  With
 * advance_counter (a device unsigned, zero before the first call) the launch
 * also advances step[0] by delta once every block has read it, in place of a
 * following fdtd_advance; the counter is left at zero.  No reference
 * counterpart. */
#define FDTD_STAGE_PLANES_MAX 8
typedef struct fdtd_stage_plane {
    const int *indices;  /* (nsteps) */
    float *stage;        /* (T, 6, sx*sy*sz) */
    int nsteps, T, x0, y0, z0, sx, sy, sz, exact;
} fdtd_stage_plane;
int fdtd_record_stage_many(const float *E0, const float *E1, const float *H0, const float *H1,
                           int *step, const fdtd_stage_plane *planes, int nplanes, int nx,
                           int ny, int nz, int pitch_z, unsigned *advance_counter, int delta,
                           void *stream);
/* Two consecutive steps' staging in one launch (the time-blocked step's
 * pair): fields[0..3] = (E0, E1, H0, H1) as fdtd_record_stage_many takes them
 * for step t = step[0], fields[4..7] for step t + 1; step[0] advances by 2
 * after every block has read it (advance_counter required).  The caller folds
 * no plane between the two steps: every plane's T is even and the pair starts
 * on an even step.  No reference counterpart. */
int fdtd_record_stage_pair(const float *const *fields, int *step, const fdtd_stage_plane *planes,
                           int nplanes, int nx, int ny, int nz, int pitch_z,
                           unsigned *advance_counter, void *stream);

/* Fold the steps staged since the last fold into the phasors, in time order:
 * run after fdtd_advance once every T steps and after the last step.  With
 * s = step[0] (steps completed) the window is [T * floor((s - 1) / T), s).
 * For each step t of the window with indices[t] >= 0 and each frequency k
 * with w = weights[k, t] != 0: phasor[k, c, i] += w * stage[t % T, c, i]
 * (float64, the same operation sequence as fdtd_record_phasor64, so the
 * result is bitwise identical). */
int fdtd_dft_fold(const int *step, const int *indices, int nsteps, const float *weights,
                  int nfreq, const float *stage, int T, double *phasor, long long count,
                  void *stream);

/* ---------------------------------------------------------------------------
 * 4. CNN surrogate (no reference counterpart: the reference optimises with
 *    the adjoint alone).  A 2-D encoder-decoder maps a design density to the
 *    modal transmission at several wavelengths and to the transmission
 *    gradient map; the design loop uses it to propose updates that a full
 *    FDTD forward accepts or rejects.  bf16 storage, float32 accumulation.
 *    Activations are NHWC (pixel p = (b*H + y)*W + x, channel fastest) with a
 *    row stride ld in elements; im2col column k = tap*C + c, tap = (dy+1)*3 +
 *    (dx+1).  bf16 buffers are passed as void pointers.
 * ------------------------------------------------------------------------ */

/* C[M, N] = A[M, K] . B[N, K]^T on the tcgen05 tensor cores (128 x BN tiles,
 * BN = 32, 64 or 128 picked from N, TMA-staged operands, float32 accumulator
 * in tensor memory).  A and B are bf16, K contiguous, 16-byte aligned, row
 * strides lda, ldb multiples of 8; rows and K columns past M, N, K read as
 * zero.  C is float32 (c_bf16 = 0) or bf16 (c_bf16 = 1, round to nearest
 * even) with row stride ldc; epilogue: + bias[n] (if bias), + C (accumulate,
 * float32 only), max(., 0) (relu).  splits > 1 divides K over that many
 * blocks (fewer when K has fewer 64-wide chunks; fdtd_sg_gemm_splits gives
 * the count used), each writing its float32 partial at C + z*split_stride,
 * with no bias, relu or accumulate: sum them with fdtd_sg_splitk_reduce.
 * layout picks the shared-memory operand layout: 0 = 128-byte swizzled rows
 * (one TMA box per operand and stage), 1 = interleaved 8 x 16-byte core
 * matrices (eight narrow boxes); results are identical. */
typedef struct fdtd_sg_gemm_args {
    const void *A;
    int lda;
    const void *B;
    int ldb;
    void *C;
    int ldc;
    int c_bf16;
    const float *bias;
    int M, N, K;
    int splits;
    long long split_stride;
    int accumulate;
    int relu;
    int layout;
} fdtd_sg_gemm_args;
int fdtd_sg_gemm(const fdtd_sg_gemm_args *args, void *stream);
/* Number of K splits fdtd_sg_gemm uses for these arguments. */
int fdtd_sg_gemm_splits(const fdtd_sg_gemm_args *args);
/* Copies the GEMM wait status to *out (0: every bounded mbarrier wait
 * completed; 1: one ran out and its tile was not written); reset != 0 clears
 * it.  Synchronous. */
int fdtd_sg_status(int *out, int reset);

/* col[p, tap*C + c] = x[p + offset(tap), c] with zero padding (3 x 3, same
 * size); columns past 9*C are left untouched. */
int fdtd_sg_im2col(const void *x, int ldx, int B, int H, int W, int C, void *col, int ldcol,
                   void *stream);
/* dst[c, r] = src[r, c] (bf16). */
int fdtd_sg_transpose(const void *src, int lds, long long rows, int cols, void *dst,
                      long long ldd, void *stream);
/* Adjoint of im2col: dx[p, c] (+)= sum over taps of dcol[p - offset(tap), tap*C + c]. */
int fdtd_sg_col2im(const float *dcol, int ldd, int B, int H, int W, int C, float *dx, int ldx,
                   int accumulate, void *stream);
/* dz = bf16(y > 0 ? dy : 0) and bias_grad[c] = sum_p of the same masked values
 * (scratch: FDTD_SG_SCRATCH_ROWS * C floats). */
#define FDTD_SG_SCRATCH_ROWS 1024
int fdtd_sg_relu_backward(const float *dy, int lddy, const void *y, int ldy, long long P, int C,
                          void *dz, int ldz, float *bias_grad, float *scratch, void *stream);
/* 2 x 2 average pool of an H x W map (H, W even) and its adjoint. */
int fdtd_sg_pool(const void *x, int ldx, int B, int H, int W, int C, void *y, int ldy,
                 void *stream);
int fdtd_sg_pool_backward(const float *dy, int lddy, int B, int H, int W, int C, float *dx,
                          int ldx, int accumulate, void *stream);
/* Nearest 2x upsample of an H x W map and its adjoint (H, W: the small map). */
int fdtd_sg_upsample(const void *x, int ldx, int B, int H, int W, int C, void *y, int ldy,
                     void *stream);
int fdtd_sg_upsample_backward(const float *dy, int lddy, int B, int H, int W, int C, float *dx,
                              int ldx, int accumulate, void *stream);
/* Transmission head: feat[b, c] = mean_p x[b, p, c]; out[b, k] = bl[k] +
 * sum_c feat[b, c] * Wl[k, c] (float32 Wl [K, C]); and its reverse mode. */
int fdtd_sg_gap_linear(const void *x, int ldx, int B, int npix, int C, const float *Wl,
                       const float *bl, int K, float *feat, float *out, void *stream);
int fdtd_sg_gap_linear_backward(const float *dout, const float *feat, const float *Wl, int B,
                                int npix, int C, int K, float *dWl, float *dbl, float *dx,
                                int ldx, int accumulate, void *stream);
/* Gradient-map head: out[p] = bg + sum_c x[p, c] * wg[c]; and its reverse
 * mode (dx overwritten; scratch: FDTD_SG_SCRATCH_ROWS * C floats). */
int fdtd_sg_head(const void *x, int ldx, long long P, int C, const float *wg, const float *bg,
                 float *out, void *stream);
int fdtd_sg_head_backward(const float *dout, const void *x, int ldx, long long P, int C,
                          const float *wg, float *dx, int lddx, float *dwg, float *dbg,
                          float *scratch, void *stream);
/* grad = scale * 2 * (pred - target); partial[i] = sum of squared
 * differences of block i (ceil(n / 256) blocks). */
int fdtd_sg_mse(const float *pred, const float *target, long long n, float scale, float *grad,
                float *partial, void *stream);
/* One Adam step (step >= 1: bias corrections 1 - b^step). */
int fdtd_sg_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1,
                 float b2, float eps, int step, void *stream);
/* bf16 copies of a float32 [cout, kw] weight: wb [cout, ldw], wt [kw, cout]
 * (wt may be NULL). */
int fdtd_sg_cast_weights(const float *w, int cout, int kw, void *wb, int ldw, void *wt,
                         void *stream);
/* out = sum_z part[z] (z ascending) for [M, N] partials split_stride apart;
 * transpose != 0 writes out[n, m]. */
int fdtd_sg_splitk_reduce(const float *part, int splits, long long stride, int M, int N, int ldp,
                          float *out, int ldo, int transpose, void *stream);
int fdtd_sg_to_bf16(const float *x, void *y, long long n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* WARP_FDTD_B200_H */
