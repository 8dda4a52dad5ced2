/* fdtd_capi.h -- C-ABI of the B200 FDTD (Yee) solver (libgdiamond_b200.so).
 *
 * The drop-in boundary for gDiamond's GPU update path.  In the reference every GPU variant is
 * a member function of the header-only class gdiamond::gDiamond that allocates device memory,
 * copies the 12 coefficient arrays in, runs T steps and copies the 6 fields out, all on the
 * legacy default stream (e.g. update_FDTD_gpu_2D, gDiamond/gdiamond_gpu.cuh:483-648;
 * update_FDTD_gpu_3D_warp_underutilization_fix, gDiamond/gdiamond_gpu.cuh:809-950;
 * update_FDTD_mix_mapping_gpu_ver3, gDiamond/gdiamond_gpu_mm_ver3.cuh:478-740).  Here the same
 * work is split into plain C calls on an opaque handle that keeps device state between calls;
 * include/gdiamond_compat.hpp rebuilds the reference class surface on top of them.
 *
 * Conventions
 *  - Grid layout on the host: x-fastest structure of arrays, idx = i + j*Nx + k*Nx*Ny, FP32.
 *  - Field components: FDTD_EX..FDTD_HZ.  Coefficient arrays (12, in this order):
 *    Cax Cay Caz Cbx Cby Cbz Dax Day Daz Dbx Dby Dbz  (gDiamond/gdiamond.hpp:891-904).
 *  - One step = the E update of all interior cells followed by the H update of all interior
 *    cells (gDiamond/gdiamond.hpp:1193-1221).  Cells on the six outer faces are never updated
 *    (they keep their value, zero unless set), as in every reference path.
 *  - Calls return fdtd_status and never exit or trap.  fdtd_last_error() gives the reason.
 *  - A handle is not thread-safe; distinct handles are independent.
 *  - fdtd_step is asynchronous on the given stream; fdtd_get_* synchronise.
 */
#ifndef GDIAMOND_B200_FDTD_CAPI_H
#define GDIAMOND_B200_FDTD_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_handle fdtd_handle;

typedef enum fdtd_status {
  FDTD_OK = 0,
  FDTD_ERR_INVALID_ARG = 1,
  FDTD_ERR_OOM = 2,
  FDTD_ERR_CUDA = 3,
  FDTD_ERR_UNSUPPORTED = 4,
  FDTD_ERR_DEVICE_TIMEOUT = 5,
  FDTD_ERR_NUMERIC = 6
} fdtd_status;

typedef enum fdtd_component {
  FDTD_EX = 0, FDTD_EY = 1, FDTD_EZ = 2, FDTD_HX = 3, FDTD_HY = 4, FDTD_HZ = 5
} fdtd_component;

/* Current-source components: J enters the E update as -J*dx, M the H update as -M*dx
 * (gDiamond/gdiamond.hpp:1198-1218). */
typedef enum fdtd_source_component {
  FDTD_JX = 0, FDTD_JY = 1, FDTD_JZ = 2, FDTD_MX = 3, FDTD_MY = 4, FDTD_MZ = 5
} fdtd_source_component;

typedef enum fdtd_source_kind {
  FDTD_SRC_POINT = 0,   /* one cell (i, j, k) */
  FDTD_SRC_PLANE_Z = 1  /* every interior cell of the z-plane k (a current sheet) */
} fdtd_source_kind;

/* Kernel families.  AUTO picks TILED when the coefficients compress to a material table,
 * else NAIVE. */
typedef enum fdtd_kernel {
  FDTD_KERNEL_AUTO = 0,
  FDTD_KERNEL_NAIVE = 1,      /* one thread per cell, separate E and H launches per step */
  FDTD_KERNEL_TILED = 2,      /* z-streaming temporally tiled kernel, BLT steps per launch;
                                 the autotuner picks the family below */
  FDTD_KERNEL_TILED_W32 = 3,  /* tiled, one cell per thread (32-wide warp rows) */
  FDTD_KERNEL_TILED_W64 = 4,  /* tiled, an x-pair of cells per thread (64-wide warp rows) */
  FDTD_KERNEL_TILED_W32P = 5  /* tiled, an x-pair per thread, two 32-wide rows per warp */
} fdtd_kernel;

/* Field storage in HBM.  F32/F16/BF16/F16E update in FP32 arithmetic; F16/BF16 store each
 * component with a per-component power-of-two scale (value = stored * scale) and run the tiled
 * x-pair kernel only.  F16E stores the E components in FP16 (scaled) and the H components in
 * FP32: 36 field bytes per cell-update instead of 24 (F16) or 48 (F32), and half of F16's
 * storage roundings per pass.  F64 stores and updates in FP64 with the naive
 * kernel: the error reference for reduced-precision runs (coefficients and waveforms widened
 * from FP32).  The reference stores float fields only (gDiamond.h). */
typedef enum fdtd_storage {
  FDTD_STORE_F32 = 0,
  FDTD_STORE_F16 = 1,
  FDTD_STORE_BF16 = 2,
  FDTD_STORE_F64 = 3,
  FDTD_STORE_F16E = 4
} fdtd_storage;

typedef struct fdtd_desc {
  int64_t nx, ny, nz;   /* grid cells per axis, each >= 3 */
  float dx;             /* spacing used in the -J*dx / -M*dx source terms */
  int32_t device;       /* CUDA device ordinal */
  int32_t storage;      /* fdtd_storage */
  int32_t kernel;       /* fdtd_kernel */
  int32_t blt;          /* time steps per tiled launch; 0 = autotuned */
  int32_t tile_rows;    /* tiled-kernel rows per tile (8, 16, 20, 24, 32 or 48); 0 = autotuned */
  int32_t z_chunks;     /* tiled-kernel z-chunks per column; 0 = autotuned */
  int32_t min_blocks;   /* tiled x-pair family: CTAs per SM the registers must allow (1, 2 or
                           4); 0 = autotuned */
} fdtd_desc;

typedef struct fdtd_source {
  int32_t component;    /* fdtd_source_component */
  int32_t kind;         /* fdtd_source_kind */
  int64_t i, j, k;      /* cell (point) or plane index k (plane) */
} fdtd_source;

/* Library version string. */
const char* fdtd_version(void);
const char* fdtd_status_string(fdtd_status s);
/* Last error message of a handle (or of the last failed fdtd_create when h == NULL). */
const char* fdtd_last_error(const fdtd_handle* h);

/* Allocates device state for one grid: two field sets, zeroed (replaces the cudaMalloc /
 * cudaMemset block of gDiamond/gdiamond_gpu.cuh:492-543). */
fdtd_status fdtd_create(const fdtd_desc* desc, fdtd_handle** out);
fdtd_status fdtd_destroy(fdtd_handle* h);

/* Per-cell coefficients from 12 host arrays of Nx*Ny*Nz floats (the H2D copies of
 * gDiamond/gdiamond_gpu.cuh:548-559).  The device deduplicates them into a material map
 * (uint16 per cell) plus a coefficient table when at most 65536 distinct 12-tuples occur;
 * otherwise the per-cell arrays are kept and the naive kernel is used. */
fdtd_status fdtd_set_coefficients(fdtd_handle* h, const float* const* coef12);
/* Same, from 12 device arrays already resident in HBM (unpitched, Nx*Ny*Nz floats each). */
fdtd_status fdtd_set_coefficients_device(fdtd_handle* h, const float* const* coef12_dev);
/* Number of distinct materials found (0 when the per-cell arrays are in use). */
fdtd_status fdtd_material_count(const fdtd_handle* h, int32_t* nmat);
/* The coefficients of gDiamond's constructor (gDiamond/gdiamond.hpp:20-73 calling
 * set_FDTD_matrices_3D_structure, gDiamond/utils.h:542-690) for a per-cell relative
 * permittivity, computed on the GPU with the reference's arithmetic (bit-identical arrays):
 * a graded pseudo-PML of t_pml cells on every face, time step dt, source omega omega0 (the
 * reference's defaults are t_pml = 10, dt = 0.05, omega0 = 2*pi), spacing = desc.dx.
 * eps_re: host array of Nx*Ny*Nz floats, or NULL for vacuum.  Then compressed as in
 * fdtd_set_coefficients. */
fdtd_status fdtd_set_permittivity(fdtd_handle* h, const float* eps_re, int32_t t_pml, float dt,
                                  float omega0);
/* Copies the per-cell coefficients last set (12 host arrays of Nx*Ny*Nz floats). */
fdtd_status fdtd_get_coefficients(fdtd_handle* h, float* const* coef12_out);

/* Replaces the source list.  waveforms = nsrc rows of T_wave FP32 samples; sample t drives
 * step t of the run (replaces the per-step 4-byte cudaMemcpy of the source value,
 * gDiamond/gdiamond_gpu.cuh:568-570).  Steps t >= T_wave see zero.  At most 8 sources. */
fdtd_status fdtd_set_sources(fdtd_handle* h, const fdtd_source* sources, int32_t nsrc,
                             const float* waveforms, int64_t T_wave);

/* Adds a running-DFT monitor on the z-plane k of one field component (the reference's
 * update_field_FFT_xy, gDiamond/kernels.cuh:87-113, here with FP64 sums): after each step t
 *   re[f][j][i] += (F(i,j,k) * cos(ph)) * scale,  im[f][j][i] -= (F(i,j,k) * sin(ph)) * scale,
 *   ph = (2*pi*freqs[f]) * ((double)t * dt).
 * At most 4 monitors, 64 frequencies each.  Writes the monitor id. */
fdtd_status fdtd_add_dft_monitor(fdtd_handle* h, int32_t component, int64_t k,
                                 const double* freqs, int32_t nf, double scale, double dt,
                                 int32_t* monitor_id);

/* Poynting flux monitor on the E plane z = k (1 <= k <= Nz-2), at nf frequencies (FP64 Hz, in
 * units of 1/dt's time unit), for a transmission spectrum.  The reference has no flux monitor,
 * only the per-cell running DFT of one component (update_field_FFT_xy,
 * gDiamond/kernels.cuh:87-113); this adds six such DFTs (monitor slots): Ex and Ey of plane k,
 * Hx and Hy of planes k-1 and k.  Co-location: in the plane Ex and Hy share (i+1/2, j), Ey and Hx
 * share (i, j+1/2); H is averaged over planes k-1 and k (z = k -+ 1/2).  Time: H of step t is
 * phased at (t + 1/2) dt, E at t dt (Yee staggering).  fdtd_get_flux then gives, per frequency,
 *   flux(f) = dx^2 * sum over the plane of Re[ Ex conj(Hy) - Ey conj(Hx) ]
 * with X(f) = sum_t x(t) exp(-i 2 pi f t'), reduced on the GPU in FP64 (fixed order).
 * fdtd_flux_monitor_ids gives the six monitor ids (their sums via fdtd_get_dft). */
fdtd_status fdtd_add_flux_monitor(fdtd_handle* h, int64_t k, const double* freqs, int32_t nf,
                                  double dt, int32_t* flux_id);
fdtd_status fdtd_get_flux(fdtd_handle* h, int32_t flux_id, double* flux_out);
/* Same into device memory (nf doubles), asynchronous on stream (or the handle's stream). */
fdtd_status fdtd_get_flux_device(fdtd_handle* h, int32_t flux_id, double* flux_dev,
                                 void* stream);
fdtd_status fdtd_flux_monitor_ids(const fdtd_handle* h, int32_t flux_id, int32_t* ids6);

/* Convolutional PML (CPML) absorbing layers in place of the reference's graded pseudo-PML
 * (gDiamond/utils.h:585-660, a real stretch folded into Ca/Cb/Da/Db in front of PEC faces).  In
 * the layers every spatial difference d of the curl becomes d / kappa + psi with the recursive
 * convolution psi <- b psi + a d, b = exp(-(sigma / kappa + alpha) dt),
 * a = sigma (b - 1) / (sigma kappa + kappa^2 alpha), on the complex-frequency-shifted stretch
 * s = kappa + sigma / (alpha + i w) (normalised units: eps0 = mu0 = c = 1).  Grading over the
 * layer depth rho in [0, 1]: sigma = sigma_max rho^order with
 * sigma_max = -(order + 1) ln(reflection) / (2 thickness dx), kappa = 1 + (kappa_max - 1)
 * rho^order, alpha = alpha_max (1 - rho); E differences use rho at integer positions, H
 * differences at half-integer ones.  Outside the layers the update is the reference's, bit for
 * bit.  Give the interior material's coefficients (e.g. fdtd_set_permittivity with t_pml = 0):
 * the CPML replaces the grading.  FP32 storage only; the psi fields live only in the slabs of
 * their axis.  With layers on, fdtd_step runs the tiled kernel over the whole grid and a shell
 * companion that recomputes, per tiled launch of k steps, the cells the layers can reach within
 * those steps (when the cells more than 3k from the layers are at least 40 % of the grid and the
 * handle's kernel is not FDTD_KERNEL_NAIVE); otherwise one E and one H kernel per step over the
 * grid.  Both give the same fields and monitor sums bit for bit.  fdtd_batch_step advances a
 * batch whose simulations all have layers with one E and one H launch per step over every
 * grid.  NULL turns the layers off. */
typedef struct fdtd_cpml_desc {
  int32_t thickness;   /* cells per face (L); each axis with layers needs >= 2 L + 2 cells */
  int32_t faces;       /* bit mask of faces with a layer: 1 -x, 2 +x, 4 -y, 8 +y, 16 -z, 32 +z */
  float order;         /* polynomial grading (3) */
  float reflection;    /* normal-incidence reflection the grading aims at (1e-6) */
  float kappa_max;     /* real stretch at the outer edge (1: none) */
  float alpha_max;     /* CFS shift at the inner edge (0.05 in units of 1/time) */
  float dt;            /* time step of the run (the reference's 0.05) */
} fdtd_cpml_desc;
fdtd_status fdtd_set_cpml(fdtd_handle* h, const fdtd_cpml_desc* desc);
/* The layers' auxiliary state, for checkpoint / resume (no reference counterpart): psi array q,
 * 0..5 of the E updates (exy exz eyz eyx ezx ezy), 6..11 of the H updates (hxz hxy hyx hyz hzy
 * hzx), FP32 in the slabs of its axis; *bytes = its size.  Synchronous; INVALID_ARG without
 * layers. */
fdtd_status fdtd_cpml_psi_bytes(const fdtd_handle* h, int32_t q, int64_t* bytes);
fdtd_status fdtd_get_cpml_psi(fdtd_handle* h, int32_t q, void* host_out);
fdtd_status fdtd_set_cpml_psi(fdtd_handle* h, int32_t q, const void* host_in);
/* The tabulated profile of one axis (0 x, 1 y, 2 z) at E positions (h_positions = 0) or H
 * positions (1): b, a, 1/kappa and the psi slot (-1 outside the layer), Nx/Ny/Nz entries each
 * (any pointer may be NULL). */
fdtd_status fdtd_get_cpml_profile(const fdtd_handle* h, int32_t axis, int32_t h_positions,
                                  float* b, float* a, float* inv_kappa, int32_t* slot);

/* Zeroes the fields and the monitor sums and sets the step counter to 0. */
fdtd_status fdtd_reset(fdtd_handle* h);
/* Runs T steps (asynchronous).  stream = a cudaStream_t, or NULL for the handle's stream. */
fdtd_status fdtd_step(fdtd_handle* h, int64_t T, void* stream);
/* Waits for the handle's work and reports any device-side error: a bounded wait that gave up
 * (FDTD_ERR_DEVICE_TIMEOUT), or a field value stored in FP16/BF16 that overflowed to +-inf or
 * became NaN because its storage scale is too small (FDTD_ERR_NUMERIC).  The reference has no
 * error path here (CUDACHECK exits, gDiamond/gdiamond_gpu.cuh:11-20). */
fdtd_status fdtd_sync(fdtd_handle* h);
/* Global step counter (number of steps run since create/reset). */
fdtd_status fdtd_get_step(const fdtd_handle* h, int64_t* t);

/* Field and monitor transfer (synchronous).  Host arrays are Nx*Ny*Nz floats (fields) and
 * nf*Nx*Ny doubles (monitor re/im, [f][j][i]). */
fdtd_status fdtd_get_field(fdtd_handle* h, int32_t component, float* host_out);
fdtd_status fdtd_set_field(fdtd_handle* h, int32_t component, const float* host_in);
fdtd_status fdtd_get_dft(fdtd_handle* h, int32_t monitor_id, double* re, double* im);
/* Checkpoint / resume (no reference counterpart: gDiamond restarts every run from zero).  With
 * the raw field planes (fdtd_get/set_planes_device) these restore a handle's whole state: the
 * step counter (which indexes the source waveforms and the DFT phase) and a monitor's sums
 * ([nf][Ny][Nx] doubles each, host buffers). */
fdtd_status fdtd_set_step(fdtd_handle* h, int64_t t);
fdtd_status fdtd_set_dft(fdtd_handle* h, int32_t monitor_id, const double* re, const double* im);
/* Device-to-device copy of a monitor's running sums into [nf][Ny][Nx] double arrays on
 * `stream` (a cudaStream_t or NULL for the handle's stream; asynchronous).  No reference
 * counterpart: gDiamond reads its DFT sums on the host only. */
fdtd_status fdtd_get_dft_device(fdtd_handle* h, int32_t monitor_id, double* re_dev,
                                double* im_dev, void* stream);
/* Raw copies of the z-planes [k0, k0+nk) of one component of the current field set between the
 * handle and an unpitched device buffer of nk*Ny*Nx values in the storage format (esz bytes
 * each, fdtd_component_bytes), on `stream` (NULL: the handle's stream; asynchronous).  The halo
 * exchange of a grid split into z-slabs (gdiamond_b200/slabs.py).  No reference counterpart:
 * gDiamond runs one grid on one GPU. */
fdtd_status fdtd_get_planes_device(fdtd_handle* h, int32_t component, int64_t k0, int64_t nk,
                                   void* dev_out, void* stream);
fdtd_status fdtd_set_planes_device(fdtd_handle* h, int32_t component, int64_t k0, int64_t nk,
                                   const void* dev_in, void* stream);
fdtd_status fdtd_storage_bytes(const fdtd_handle* h, int32_t* esz);
/* Bytes per stored value of one component (0..5 = Ex Ey Ez Hx Hy Hz): differs from
 * fdtd_storage_bytes only for F16E (2 for E, 4 for H); the raw plane copies above move values
 * of this size.  No reference counterpart. */
fdtd_status fdtd_component_bytes(const fdtd_handle* h, int32_t component, int32_t* esz);
/* Device-to-device field copy into an unpitched Nx*Ny*Nz float array (asynchronous). */
fdtd_status fdtd_get_field_device(fdtd_handle* h, int32_t component, float* dev_out,
                                  void* stream);

/* Per-component storage scale for components stored in FP16/BF16 (ignored for FP32/FP64 ones,
 * so F16E uses scale6[0..2] only); default 1.  Each scale is rounded to the nearest power of
 * two, so scaling never rounds. */
fdtd_status fdtd_set_storage_scale(fdtd_handle* h, const float* scale6);
/* Field transfer into FP64 host memory (any storage; exact for F64 storage). */
fdtd_status fdtd_get_field_f64(fdtd_handle* h, int32_t component, double* host_out);

/* Kernel configuration actually used by the last fdtd_step: out = {kernel, blt, tile_rows,
 * z_chunks, launches in the last fdtd_step, min_blocks}; kernel is FDTD_KERNEL_NAIVE,
 * _TILED_W32, _TILED_W64 or _TILED_W32P. */
fdtd_status fdtd_get_config(const fdtd_handle* h, int32_t* out6);
/* DFT fold launches of the last fdtd_step or fdtd_batch_step that advanced h.  The tiled
 * kernels stage monitor-plane values in a ring of 128 steps per monitor and a fold kernel adds
 * them to the FP64 sums (bit-identical to accumulating every step) before the ring wraps and
 * at the end of the call, so the sums are complete when the step call's work has run.  No
 * reference counterpart: gDiamond accumulates its monitors with one kernel per step. */
fdtd_status fdtd_dft_folds(const fdtd_handle* h, int32_t* n);

/* Test hook for the failure path (no reference counterpart: the reference's CUDACHECK prints
 * and exits, gDiamond/gdiamond_gpu.cuh:11-20).  In the next tiled fdtd_step launch only, tile
 * (bx, by, bz) of the launch grid does not issue the shared-memory copy of its z-iteration
 * `iteration`, and every bounded wait of that launch gives up after wait_cycles SM clocks
 * instead of about a second.  The tile's wait for that copy then runs out: the tile leaves its
 * z-march after its copies in flight have landed, nothing faults or hangs, and fdtd_sync returns
 * FDTD_ERR_DEVICE_TIMEOUT (the fields are invalid; fdtd_reset makes the handle usable again).
 * Single-grid steps only (not batches). */
fdtd_status fdtd_debug_fail_copy(fdtd_handle* h, int32_t bx, int32_t by, int32_t bz,
                                  int32_t iteration, int64_t wait_cycles);

/* Uniform-material fast path of the tiled x-pair kernels (on by default).  When the material
 * held by the most cells is isotropic and lossless (Ca = Da = 1, one Cb and one Db on all three
 * axes: vacuum or a plain dielectric), warps whose cells all hold it, lie off the grid faces
 * and hold no source update E' = E + Cb*curl H, H' = H + Db*curl E with paired FP32
 * instructions and the two coefficients in registers.  Since 1*x == x the results are those of
 * the general per-cell path bit for bit; enable = 0 forces the general path (for comparison).
 * No reference counterpart: gDiamond reads all 12 coefficient arrays for every cell and step
 * (gDiamond/kernels.cuh:337-394).  fdtd_fast_path reports whether the path is in use. */
fdtd_status fdtd_set_fast_path(fdtd_handle* h, int32_t enable);
fdtd_status fdtd_fast_path(const fdtd_handle* h, int32_t* active);

/* Builds a material map from 12 device coefficient arrays without allocating anything.
 * No counterpart in the reference (which keeps 12 per-cell arrays); it is the allocation-free
 * form of the deduplication that fdtd_set_coefficients runs, for callers that cannot allocate
 * device memory at that point: an application that owns all device memory through its own
 * pool, a loop where cudaMalloc's implicit synchronisation is not acceptable, or code that
 * must not grow its footprint after start-up.
 *   coef12_dev   12 device arrays of nx*ny*nz floats (unpitched, Cax..Dbz)
 *   mat_dev      out: nx*ny*nz uint16 material ids (device)
 *   table_dev    out: max_materials x 12 floats (device), row id = the tuple Cax..Dbz
 *   nmat_out     out (host): number of distinct tuples found
 * Limit: at most 4096 distinct tuples; max_materials > 4096 is rejected with
 * FDTD_ERR_INVALID_ARG, data with more distinct tuples than max_materials with
 * FDTD_ERR_UNSUPPORTED (such data is rejected after a short pass).  The scratch is a fixed
 * ~1.25 MB device array that every GPU loading the library holds until exit; all calls share
 * it (each clears it first), so calls that overlap on the GPU race.  The first call on each
 * device resolves that array's address.  The call synchronises `stream` (a cudaStream_t or
 * NULL), so it cannot be made on a stream that is being captured.  Ids follow table-slot order
 * assigned by atomics: the numbering may differ between calls (map and table always agree). */
fdtd_status fdtd_build_material_map_noalloc(const float* const* coef12_dev, int64_t nx,
                                            int64_t ny, int64_t nz, uint16_t* mat_dev,
                                            float* table_dev, int32_t max_materials,
                                            int32_t* nmat_out, void* stream);

/* ---------------------------------------------------------------- batches
 * Many independent simulations advanced together.  The reference runs one grid per call;
 * here a batch groups existing handles (same device and storage, coefficients compressed to a
 * material map, CPML layers on all of them or on none) and fdtd_batch_step advances all of them
 * with one persistent launch of the tiled x-pair kernel per BLT steps: CTAs pull (simulation,
 * tile) work items, longest first, from an atomic queue, so grids of uneven size share the GPU
 * without per-grid launches.  A batch with CPML layers instead runs one E and one H launch per
 * step over every grid. */
typedef struct fdtd_batch fdtd_batch;

fdtd_status fdtd_batch_create(fdtd_handle* const* sims, int32_t n, fdtd_batch** out);
fdtd_status fdtd_batch_destroy(fdtd_batch* b);
/* Advances every simulation of the batch by T steps from its own state (step counter, fields,
 * sources, monitors).  use_graph != 0: the launch sequence is captured in a CUDA graph the
 * first time and replayed while (T, each simulation's step counter and field set) repeat.
 * stream: a cudaStream_t or NULL for the batch's own stream. */
fdtd_status fdtd_batch_step(fdtd_batch* b, int64_t T, int32_t use_graph, void* stream);
/* out = {blt, tile_rows, persistent CTAs, work items per launch (tile columns x z-chunks),
 * launches in the last step, 1 if the last step replayed a graph}. */
fdtd_status fdtd_batch_get_config(const fdtd_batch* b, int32_t* out6);
const char* fdtd_batch_last_error(const fdtd_batch* b);

/* ---------------------------------------------------------------- spectrum surrogate
 * No reference counterpart (gDiamond has no learned component).  An ensemble of `members`
 * MLPs dims[0] -> dims[1] -> ... -> dims[n_dims-1], GELU between layers, mean-squared-error
 * loss, trained with Adam on the GPU.  FP32 master weights, BF16 GEMM operands, FP32
 * accumulation on the tensor cores; all members run in the same launches.
 *
 * Parameter layout of one member (fdtd_mlp_layout): for every layer l, W_l row-major
 * [dims[l+1]][dims[l]] at w_off[l] and b_l [dims[l+1]] at b_off[l] (blocks start on multiples
 * of 8 floats; gaps are zero).  get/set_params move all members: [members][n_params]. */
typedef struct fdtd_mlp fdtd_mlp;

/* GEMM path of an ensemble: tcgen05.mma with the accumulator in tensor memory, the warp-level
 * mma.sync kernel (the same products), or AUTO (default): tcgen05 for products of >= 1024
 * rows (inference), mma.sync for the short minibatch products of training. */
typedef enum fdtd_mlp_gemm {
  FDTD_MLP_GEMM_TCGEN05 = 0,
  FDTD_MLP_GEMM_MMA_SYNC = 1,
  FDTD_MLP_GEMM_AUTO = 2
} fdtd_mlp_gemm;

fdtd_status fdtd_mlp_create(const int32_t* dims, int32_t n_dims, int32_t members, uint64_t seed,
                            int32_t device, fdtd_mlp** out);
fdtd_status fdtd_mlp_destroy(fdtd_mlp* m);
const char* fdtd_mlp_last_error(const fdtd_mlp* m);
fdtd_status fdtd_mlp_set_gemm(fdtd_mlp* m, int32_t kind);
/* n_params per member; w_off / b_off (may be NULL) receive n_dims-1 offsets each. */
fdtd_status fdtd_mlp_layout(const fdtd_mlp* m, int64_t* n_params, int64_t* w_off, int64_t* b_off);
fdtd_status fdtd_mlp_get_params(fdtd_mlp* m, float* out);
/* Replaces all members' parameters and restarts Adam. */
fdtd_status fdtd_mlp_set_params(fdtd_mlp* m, const float* in);
/* Training set (host): x [n][dims[0]], y [n][dims[last]], copied to the device. */
fdtd_status fdtd_mlp_set_data(fdtd_mlp* m, const float* x, const float* y, int64_t n);
/* Loss (mean squared error, per member) and gradient of every member on one batch (host x, y
 * shared by all members); grads (may be NULL) [members][n_params]. */
fdtd_status fdtd_mlp_grad(fdtd_mlp* m, const float* x, const float* y, int64_t n, float* loss,
                          float* grads);
/* `epochs` passes over the training set, minibatches of `batch` rows, every member its own
 * shuffle per epoch (seeded), one Adam step (b1 0.9, b2 0.999, eps 1e-8) per minibatch.
 * loss_out (may be NULL): [epochs][members] mean squared error over each epoch. */
fdtd_status fdtd_mlp_train(fdtd_mlp* m, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                           float* loss_out);
/* Ensemble mean and standard deviation over the members (host buffers, [n][dims[last]]);
 * per_member (may be NULL) [members][n][dims[last]]. */
fdtd_status fdtd_mlp_predict(fdtd_mlp* m, const float* x, int64_t n, float* mean, float* sd,
                             float* per_member);
/* The same on device buffers, ordered after and before work on `stream` (cudaStream_t). */
fdtd_status fdtd_mlp_predict_device(fdtd_mlp* m, const float* x_dev, int64_t n, float* mean_dev,
                                    float* sd_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif
