/*
 * fwt.h -- C-ABI of the B200 woven-field construction library (libfwt.so).
 *
 * The reference (FastWeavTurb, program `Weav_ver5_8_2`) is one Fortran/MPI program whose
 * seams are implicit-interface subroutines and two input files.  Each entry point below
 * replaces one of those seams; the citation names the reference code it stands in for.
 * Plain C types only: pointers, sizes, doubles.  Every function returns 0 on success and
 * a negative FWT_E_* code on error; fwt_last_error() gives the message (thread-local).
 *
 * Host arrays are caller-owned.  A 3-D field crossing this boundary is column-major
 * (x fastest), i.e. Fortran `field(nx, ny, nz)`.  Device memory is owned by the context.
 * One context per host thread; no internal locking.
 */
#ifndef FWT_H
#define FWT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FWT_OK 0
#define FWT_E_ARG (-1)      /* invalid argument */
#define FWT_E_CUDA (-2)     /* CUDA runtime / cuFFT failure */
#define FWT_E_IO (-3)       /* file missing, unreadable or malformed */
#define FWT_E_STATE (-4)    /* call out of order (e.g. statistics before velocity) */
#define FWT_E_NOMEM (-5)    /* device allocation failed or exceeds the cap */
#define FWT_E_TIMEOUT (-6)  /* a bounded device-side wait ran out */
#define FWT_E_RANGE (-7)    /* value outside the supported range */

typedef struct fwt_ctx fwt_ctx;

/* Run parameters: the scalar block of parameters_input.dat (tube.f90:190-217) plus the
 * compile-time switches of tube.f90:53-59,129 as runtime fields. */
typedef struct {
    int N;              /* grid points per side, nx = ny = nz (tube.f90:193,200-201) */
    int N_downsample;   /* field output points per side (tube.f90:195,1056) */
    int line_s, line_e; /* 1-based inclusive range of lines to deposit (tube.f90:197-199,528);
                           line_e = 0: up to the last line */
    double sigma_ratio; /* sigma_max / sigma_min (tube.f90:203,538) */
    double eta_t;       /* twist rate eta0 (tube.f90:206) */
    int ntf_times;      /* sub-segments per 2pi of turning (tube.f90:210,641) */
    int ntf_pre;        /* presamples per section (tube.f90:212,627) */
    double Rtube_ratio; /* truncation radius / sigma (tube.f90:214,790) */
    double dzeta_sup;   /* upper bound of the sigma difference step (tube.f90:217,826) */
    int precision;      /* 32: FP32 bulk arithmetic; 64: FP64 throughout */
    int deposit_mode;   /* 0: tile-owned cell-list kernel (default); 1: reference box walk */
    int device;         /* CUDA device ordinal */
    void *stream;       /* cudaStream_t to launch on, or NULL for a context-owned stream */
    int if_pdf;         /* tube.f90:57 (default 1) */
    int if_Sp;          /* tube.f90:58 (default 1) */
    int Sp_order;       /* tube.f90:58 (default 10) */
    int pdf_bins;       /* tube.f90:129 bin_num (default 1000) */
    int vorticity_output; /* tube.f90:55 (default 1) */
    size_t mem_cap;     /* bytes of device memory the context may hold (0 = no cap); a cap also
                           bounds the lines' batches (mem_cap / 24576 nodes) and the list of
                           pairs handed to FP64 (mem_cap / 256 entries) */
} fwt_params;

/* Fill *p with the reference defaults (the values of FBB_with_parameters.m:205-225 and
 * the switches of tube.f90:53-59). */
int fwt_default_params(fwt_params *p);

/* Replaces MPI_Init + set_fft_plans + wavenumber (tube.f90:161-163,306-307;
 * subroutine.f90:860-919). */
int fwt_create(const fwt_params *p, fwt_ctx **out);
/* Replaces destroy_fft_plans + the deallocations + MPI_Finalize (tube.f90:1213-1238). */
int fwt_destroy(fwt_ctx *ctx);

/* Reads both input files; the scalar block of params_path overrides N..dzeta_sup of the
 * context (tube.f90:168-223, 341-379).  Writes nothing. */
int fwt_load_inputs(fwt_ctx *ctx, const char *centerline_path, const char *params_path);
/* Read and validate the two input files without a context or a GPU (the reference's input
 * reading, tube.f90:168-223, 341-379, and the checks fwt_load_inputs and fwt_create apply):
 * p receives the file's scalars over the defaults it holds, nline and nodes the line and node
 * counts.  A truncated or non-numeric file, a non-finite coordinate, a line with fewer than two
 * nodes, a missing parameter row, N_downsample not dividing N or a bad line range is an
 * FWT_E_IO / FWT_E_ARG error naming the fault. */
int fwt_check_inputs(const char *centerline_path, const char *params_path, fwt_params *p, int *nline,
                     int64_t *nodes);

/* Array form of the same inputs (tube.f90:353-379 after the broadcasts): nline lines,
 * npoint[l] nodes each, xyz row-major (npointall x 3) host doubles in [-pi,pi), and the
 * per-line columns of parameters_input.dat (tube.f90:221-223). */
int fwt_set_centerlines(fwt_ctx *ctx, int nline, const int64_t *npoint, const double *xyz,
                        const double *sigma, const double *Gamma, const int *n_T,
                        const int *if_filter);
/* Same, with the copy asynchronous: the call returns once the upload is queued, and the
 * deposition of each batch of lines waits only for that batch's nodes, so the transfer
 * overlaps the work on the lines before them.  xyz must stay valid and unchanged until the
 * next fwt_deposit / fwt_run returns (or fwt_destroy); pinned host memory copies at the link's
 * full rate.  Results are those of fwt_set_centerlines. */
int fwt_set_centerlines_async(fwt_ctx *ctx, int nline, const int64_t *npoint, const double *xyz,
                              const double *sigma, const double *Gamma, const int *n_T,
                              const int *if_filter);
/* Same, with the node coordinates already on this context's device (x, y, z: npointall
 * doubles each).  The device arrays must stay valid until fwt_deposit returns. */
int fwt_set_centerlines_device(fwt_ctx *ctx, int nline, const int64_t *npoint, const double *d_x,
                               const double *d_y, const double *d_z, const double *sigma,
                               const double *Gamma, const int *n_T, const int *if_filter);

/* Deposit lines line_s..line_e (1-based inclusive) into omega, applying each flagged
 * line's spectral filter after it (tube.f90:392-946: centerline preprocessing, quintic
 * splines, adaptive sub-segmentation, Burgers-tube deposition, filter_spec). */
int fwt_deposit(fwt_ctx *ctx, int line_s, int line_e);
/* Sharp spectral low-pass |k|^2 > k_c^2 on omega (subroutine.f90:1225-1277). */
int fwt_filter(fwt_ctx *ctx, double k_c);
/* E(k) of omega, then spectral Biot-Savart omega -> u with the energy reduction fused
 * (tube.f90:972-1023: spectrum + fourier_forward x3 + i k x w / |k|^2 + fourier_backward x3). */
int fwt_biot_savart(fwt_ctx *ctx);
/* E, u' = sqrt(2E/3), and the scaling of omega and u by 1/u'; enstrophy after scaling
 * (tube.f90:1026-1044, cal_helicity subroutine.f90:1550-1569). */
int fwt_normalize(fwt_ctx *ctx, double *up, double *Etot, double *enstrophy);
/* Shell spectrum, nshell = N/2 values for shells 1..N/2 (subroutine.f90:1604-1638).
 * which = 0: omega before normalisation; 1: u after normalisation. */
int fwt_spectrum(fwt_ctx *ctx, int which, double *Ek, int nshell);
/* PDF with the reference's REAL(4) bin layout (subroutine.f90:1-62).  which = 0: u,
 * 1: omega; component = -1 pools the three components (tube.f90:1169-1177), 0/1/2 picks one.
 * val, pdf: nbins floats; counts (may be NULL): nbins uint64. */
int fwt_pdf(fwt_ctx *ctx, int which, int component, int nbins, float *val, float *pdf,
            uint64_t *counts);
/* The same PDF for callers that cannot allocate device memory (no counterpart in the
 * reference).  d_data: a device field of nx*ny*nz floats (precision 32) or doubles (64) on the
 * current device; values binned are (float)(x * scale); val, pdf: nbins floats, counts (may
 * be NULL): nbins uint64, all host memory.  Allocates nothing: its scratch is a static device
 * array of at most 8192 bins (about 128 KB, held by every GPU that loads the library); larger
 * nbins is rejected with FWT_E_RANGE.  The first call on a device looks up that array's
 * address and should come before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race.  stream: a cudaStream_t or NULL. */
int fwt_pdf_noalloc(const void *d_data, int precision, int nx, int ny, int nz, double scale, int nbins,
                    void *stream, float *val, float *pdf, uint64_t *counts);
/* Longitudinal structure functions S_p(r), p = 1..pmax, at nr separations r (grid units)
 * (subroutine.f90:64-129).  Sp: pmax x nr doubles, Sp[(p-1)*nr + m]. */
int fwt_sp(fwt_ctx *ctx, int pmax, const int *r, int nr, double *Sp);
/* Scaling exponents and flatness of a structure-function table, as the reference's
 * post-processing of Sp.dat (output/stat/Sp_zeta.m:3-23, output/stat/Flatness.m:14-19):
 * zeta[p-1] = least-squares slope of log|S_p| against log(rdr) over rows nr-9 .. nr-4
 * (0-based), p = 1..pmax (needs nr >= 10); flat[m] = S_4 / S_2^2 on every row (needs
 * pmax >= 4).  rdr: nr separations r*dr; Sp: pmax x nr as fwt_sp writes it.  Either output
 * may be NULL.  Host arithmetic only. */
int fwt_sp_exponents(const double *rdr, const double *Sp, int nr, int pmax, double *zeta, double *flat);
/* Downsampled |omega| and omega.u (normalised) as float32, Fortran order
 * (n_d, n_d, n_d, 2) (tube.f90:1055-1071). */
int fwt_field_wh(fwt_ctx *ctx, float *host_out);
/* Copy a normalised (after fwt_normalize) or raw field to the host as doubles,
 * column-major.  which = 0: omega, 1: u; component 0..2. */
int fwt_copy_field(fwt_ctx *ctx, int which, int component, double *host_colmajor);
/* The vortex-surface-field deviation of cal_deviation (subroutine.f90:1519-1546), whose call
 * the reference keeps commented out (tube.f90:1050-1053, 1201): the mean over the grid of
 * |omega . grad phi| / (|omega| |grad phi| + 1e-11), grad phi by sixth-order central
 * differences on the periodic grid (wall_phiv's ghost layers, subroutine.f90:1575-1601).
 * d_phi: a device scalar field N^3 of the context's precision (column-major), or NULL for
 * phi = |omega| (the "VSF deviation of vorticity magnitude" of tube.f90:1201).  0 when omega
 * is everywhere tangent to the level sets of phi. */
int fwt_vsf_deviation(fwt_ctx *ctx, const void *d_phi, double *deviation);
/* Total helicity, cal_helicity of (omega, u) (subroutine.f90:1550-1569, its call commented out
 * at tube.f90:1027): sum of omega . u times the cell volume (2 pi / N)^3, of the normalised
 * fields after fwt_normalize, of the raw fields before. */
int fwt_helicity(fwt_ctx *ctx, double *helicity);
/* Restrict the context to the z-slab of planes z0 .. z0 + nz - 1 (0-based; z0 and nz multiples
 * of 8; z0 = nz = 0 restores the whole grid): the fields become N x N x nz (column-major, plane
 * z0 first) and fwt_deposit deposits every line's contribution to those planes only -- the
 * reference's z-slab ownership (tube.f90:261-265, 800-804), for a grid split over GPUs.  Needs
 * deposit_mode 0.  The spectral and statistics entry points refuse a slab context
 * (FWT_E_STATE): the distributed driver does them across the slabs (fwt_biot_savart_block,
 * fwt_sp_block).  Clears the context's fields. */
int fwt_set_slab(fwt_ctx *ctx, int z0, int nz);
/* The Biot-Savart pass of fwt_biot_savart on one y-pencil of the half spectrum, for a grid split
 * over GPUs (the pencil transposes of the reference's fourier_forward/backward,
 * subroutine.f90:938-968, are the caller's): spec (device, the context's precision) holds three
 * components, each [N kz][ny ky][N/2 + 1 kx] for ky = y0 .. y0 + ny - 1, the unscaled forward
 * transforms of omega; in place they become u^ = i k x w^ / |k|^2 scaled by 1/N^3.  sums
 * (host, 2 (N/2 + 1) + 2 doubles) receives this pencil's shell sums of 1/2 |w^|^2 at
 * [1 .. N/2], of 1/2 |u^|^2 at [N/2 + 2 .. N + 1], and its energy and enstrophy at [N + 2],
 * [N + 3]; the caller adds them over the pencils. */
int fwt_biot_savart_block(fwt_ctx *ctx, void *spec, int y0, int ny, double *sums);
/* Structure-function sums of one velocity component on a device box n0 x n1 x n2 (x fastest,
 * the context's precision) along `axis`, whose extent must be N (a z-slab for axes 0 and 1, a
 * y-pencil for axis 2): sums[p * nr + m] = sum over the box's lines of (du scale)^(p + 1),
 * p = 0..9, du the increment at separation r[m] (Sp_calculate's sums, subroutine.f90:64-129,
 * before the division by 3 N^3). */
int fwt_sp_block(fwt_ctx *ctx, const void *u, int n0, int n1, int n2, int axis, double scale, const int *r, int nr,
                 double *sums);
/* Isosurface of |omega| on the field_wh data box, coloured by the helicity omega . u: the
 * compute part of the reference's rendering script (output/field_wh_norm.py:56-89), whose
 * rendering needs a graphics stack and is not reproduced.  The box is n_d^3 points of the
 * normalised fields (after fwt_normalize) at the script's coordinates x_i = 2 pi i / (n_d - 1).
 * iso <= 0 takes the script's iso value 3 rms(|omega|) / sqrt 2 (returned in *iso_used).
 * Marching tetrahedra: tris receives ntris triangles of 3 vertices (x, y, z, helicity), 12
 * floats per triangle, wound with the normal pointing to decreasing |omega|, in a deterministic
 * order.  tris = NULL only counts; a count above max_tris is FWT_E_RANGE. */
int fwt_isosurface(fwt_ctx *ctx, float iso, float *tris, int64_t max_tris, int64_t *ntris, float *iso_used);
/* Device address of a field held by the context: three N^3 arrays (components x, y, z, each
 * column-major, x fastest) of the context's precision (float or double), raw (unnormalised:
 * divide by u' of fwt_normalize for the normalised field).  Valid until the next call that
 * rebuilds the field or fwt_destroy; the caller must not free it.  (No counterpart in the
 * reference, whose fields are Fortran arrays of the caller; this gives zero-copy access.) */
int fwt_field_device(fwt_ctx *ctx, int which, void **ptr);
/* Write the reference's output tree under outdir: parameters_output.dat,
 * centerline_output.dat, info.dat, test_data.dat, field_wh.dat, stat/spectrum_vor_temp.dat,
 * stat/spectrum.dat, stat/pdf_um.dat, stat/pdf_wm.dat, stat/Sp.dat (tube.f90:171,226-258,
 * 519-526,623,1055-1188). */
int fwt_write_outputs(fwt_ctx *ctx, const char *outdir);
/* The whole program Weav_ver5_8_2 run in `rundir` (inputs read from it, outputs written to
 * rundir/output), equivalent to `mpirun ./tube` there (tube.f90:30-1240). */
int fwt_run_dir(const char *rundir, const fwt_params *p);
/* The path from centerlines already set on the context to all statistics on the device
 * (tube.f90:392-1188 without file output).  Host copies of the statistics are made. */
int fwt_run(fwt_ctx *ctx);

/* Per-phase device times in milliseconds of the last fwt_run / phase calls:
 * t[0] centerline set-up, t[1] deposition, t[2] Biot-Savart + spectra, t[3] statistics,
 * t[4] total.  Returns the number of values written (<= n). */
int fwt_timings(fwt_ctx *ctx, double *t, int n);
/* Device time (ms, CUDA events on the context's stream) and launch count of each kernel
 * category in the last fwt_run: 0 section presampling, 1 other centerline set-up, 2 cell-list
 * binning, 3 deposition, 4 fused Biot-Savart, 5 cuFFT, 6 statistics, 7 generator.  (The
 * reference has no counterpart; it logs phase wall times to info.dat, tube.f90:519-953.) */
int fwt_kernel_times(fwt_ctx *ctx, double *ms, int64_t *launches, int n);
/* The reference's optional field outputs, switched off there by its compile-time flags u_out
 * and d_out (tube.f90:55) and off by default here: with u_out, fwt_write_outputs also writes
 * field_uw.dat (tube.f90:1075-1100), with d_out field_wd.dat (tube.f90:1102-1120), both in the
 * raw float32 format of field_wh.dat and only when vorticity_output is set, as in the
 * reference. */
int fwt_set_outputs(fwt_ctx *ctx, int u_out, int d_out);
/* The data boxes of those files after fwt_run: field_uw -> host_out[6 * n_d^3] (ux, uy, uz, wx,
 * wy, wz, each n_d^3 in Fortran order), field_wd -> host_out[2 * n_d^3] (|omega| and the
 * dissipation S_ij S_ij of dissipation_field, subroutine.f90:1086-1126), all of the normalised
 * fields at the points i * N / n_d.  fwt_field_wd allocates, on first use, one extra half
 * spectrum and three fields of the context's precision. */
int fwt_field_uw(fwt_ctx *ctx, float *host_out);
int fwt_field_wd(fwt_ctx *ctx, float *host_out);
/* Counters of the last deposition: c[0] lines, c[1] sections, c[2] sub-segments,
 * c[3] candidate (tile, record) pairs, c[4] kernel launches of the last fwt_run, c[5] accepted
 * (grid point, sub-segment) pairs, i.e. vorticity evaluations, c[6] the pairs the FP32 path
 * handed to FP64: those with a plane test within its FP32 rounding bound (decided by the FP64
 * tests) and accepted ones with a large curved-branch amplification. */
int fwt_counters(fwt_ctx *ctx, int64_t *c, int n);

/* Tuning knobs of the context (no counterpart in the reference).  FWT_TUNE_PIECE_RT_CELLS:
 * lines whose truncation radius Rtube_ratio * sigma_max is at most `value` grid spacings are
 * deposited by the chord-piece kernel, thicker ones by the sub-segment kernel (value < 0
 * restores the default, 8).  Results agree within FP32 rounding either way; the choice is
 * speed only, and the ensemble autotuner sets it per grid size. */
#define FWT_TUNE_PIECE_RT_CELLS 1
/* FWT_TUNE_RASTER_RT_CELLS: piece lines whose truncation radius is at most `value` grid
 * spacings are rasterised once per piece (their accepted points listed before the deposition)
 * instead of searched within every tile; 0 (the default; value < 0 restores it) switches it
 * off.  The accepted points and their values are the same either way. */
#define FWT_TUNE_RASTER_RT_CELLS 2
/* FWT_TUNE_SCATTER_RT_CELLS: on the FP32 path, piece lines whose truncation radius is at most
 * `value` grid spacings are deposited without tiles: each piece is searched once and its
 * contributions are added as int64 fixed point with global reductions (the sums do not depend
 * on the order); thicker piece lines go through the tiles.  0 switches it off, value < 0
 * restores the default, 5.  The field is the same either way to FP32 rounding. */
#define FWT_TUNE_SCATTER_RT_CELLS 3
/* FWT_TUNE_DEFER_MAX_PAIRS: the most entries (16 bytes each) the list of pairs an FP32 launch
 * hands to FP64 grows to after an overflow; a launch that hands over more lists and evaluates
 * them in windows of tiles (or of pieces) that fit.  value < 1 restores the default, 2^26
 * (1 GiB), or mem_cap / 256 under a memory cap.  The field is the same, bit for bit, whatever
 * the limit. */
#define FWT_TUNE_DEFER_MAX_PAIRS 4
int fwt_set_tuning(fwt_ctx *ctx, int key, double value);

/* Message of the last error on this thread. */
int fwt_last_error(char *buf, int len);

/* ------------------------------------------------------------------ fBb generator
 * Fractional-Brownian-bridge centerlines on the device (FBB_with_parameters.m:76-126).
 * levels: nlev entries of (tubes, nodes per tube, H, dB).  Output xyz device arrays
 * sized sum(tubes*nodes); d_x/d_y/d_z must be device pointers of this context's device.
 * Tube t (global index over levels) draws from Philox stream (seed, t).  FP64 prefix sums. */
int fwt_fbb_generate(fwt_ctx *ctx, uint64_t seed, int nlev, const int *tubes, const int *nodes,
                     const double *H, const double *dB, double *d_x, double *d_y, double *d_z);
/* Circulation signs (+1/-1) of tubes [0, ntubes) for the same seed. */
int fwt_fbb_signs(uint64_t seed, int ntubes, int *signs);

/* ------------------------------------------------------------------ learned surrogate
 * No counterpart in the reference (its statistics are only plotted there).  A multilayer
 * perceptron n_in -> width (depth hidden layers, GELU) -> n_out trained with Adam on the
 * weighted mean-square error sum_j w_j (y_j - t_j)^2 / (batch n_out); its matrix products run
 * on the tensor cores (BF16 operands, FP32 accumulation), everything else in FP32.  Host
 * arrays are row-major (batch x features). */
typedef struct fwt_mlp fwt_mlp;
/* n_in 1..64, width 16..256 (multiple of 16), depth >= 1, n_out 1..256; weights drawn
 * uniform +-sqrt(6 / (fan_in + fan_out)) from seed, biases zero. */
int fwt_mlp_create(int device, int n_in, int width, int depth, int n_out, int batch_max, uint64_t seed,
                   fwt_mlp **out);
int fwt_mlp_destroy(fwt_mlp *m);
/* Parameter count and the flattened parameters, layer by layer: W (n_out_l x n_in_l,
 * row-major) then b. */
int fwt_mlp_nparams(fwt_mlp *m, int64_t *n);
int fwt_mlp_get_params(fwt_mlp *m, float *params);
int fwt_mlp_set_params(fwt_mlp *m, const float *params);
/* y = mlp(x) for batch <= batch_max rows. */
int fwt_mlp_forward(fwt_mlp *m, const float *x, int batch, float *y);
/* Loss and its gradients with respect to the parameters (fwt_mlp_get_params layout) and the
 * inputs (batch x n_in); loss, grad_params, grad_x and w_out (n_out weights) may be NULL. */
int fwt_mlp_loss_grad(fwt_mlp *m, const float *x, const float *t, const float *w_out, int batch, double *loss,
                      float *grad_params, float *grad_x);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, learning rate lr) on a batch. */
int fwt_mlp_train_step(fwt_mlp *m, const float *x, const float *t, const float *w_out, int batch, float lr,
                       double *loss);
/* The surrogate's tensor-core product on device arrays: C (M x N, FP32, leading dimension
 * ldc) = A (M x K, BF16) . B (N x K, BF16)^T, K a multiple of 64, operands 16-byte aligned. */
int fwt_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int ldc, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FWT_H */
