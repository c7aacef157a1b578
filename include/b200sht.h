/*
 * b200sht: spherical-harmonic transform pair on a Gaussian grid, B200 (sm_100a).
 *
 * C ABI for the transform calls of the ArWen Global sl_si dycore
 * (FahrenheitResearch/gpuwm-global).  Every entry point returns an int status
 * (0 = ok) and leaves a thread-local message readable with sht_last_error(),
 * the convention of rust/global-render-kernels/src/lib.rs:1-40 in the
 * reference.  Device buffers are owned by the caller and passed as plain
 * device pointers; the plan owns its Legendre tables, FFT twiddles and
 * scratch.  Work is stream-ordered on the caller's stream (a cudaStream_t
 * passed as void*, NULL = legacy default stream) with no implicit host sync.
 *
 * Layouts (the reference's, src/arwen_global/spectral/transform.py:1051-1144):
 *   grid     (planes, nlat, nlon) real, C-contiguous, row 0 southernmost
 *   spectral (planes, T+1, T+1) complex interleaved (re, im), indexed [n, m],
 *            zero above the triangle (m > n), Imag(c[n,0]) = 0 on output.
 * Element type: double/complex128 for SHT_PREC_F64 plans, float/complex64
 * for SHT_PREC_F32 and SHT_PREC_SPLIT16 plans.
 */
#ifndef B200SHT_H
#define B200SHT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHT_ABI_VERSION 1

/* Arithmetic of the Legendre contractions. */
#define SHT_PREC_F64 0     /* FP64 SIMT: the parity path (1e-12 vs FP64 reference) */
#define SHT_PREC_F32 1     /* plain FP32 FFMA path */
#define SHT_PREC_SPLIT16 2 /* FP16 hi+lo split on tcgen05 tensor cores, FP32 accumulate */

/* sht_plan_create flags (bitwise or). */
#define SHT_FLAG_GEOMETRY_ONLY 1 /* Gauss nodes and weights only */
#define SHT_FLAG_GENERIC_FFT 2   /* shared-memory Stockham FFTs even where the
                                    register-resident kernels apply (testing) */

/* Status codes. */
#define SHT_OK 0
#define SHT_ERR_ARG 1      /* invalid argument (shape, pointer, precision) */
#define SHT_ERR_CUDA 2     /* a CUDA runtime call failed */
#define SHT_ERR_DEVICE 3   /* a kernel reported an error word (bounded wait expired) */
#define SHT_ERR_STATE 4    /* plan in an unusable state */

typedef struct sht_plan sht_plan;
typedef struct sht_vertical sht_vertical;
typedef struct sht_batch sht_batch;

/* ABI version of the loaded library (SHT_ABI_VERSION). */
int sht_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* sht_last_error(void);

/* Build a plan on the current device: FP64 Gauss nodes/weights by Newton
 * iteration, the normalised P_nm recurrence, dP/dphi, the Gram-corrected
 * analysis rows and the vector-analysis tables, all computed on the GPU, then
 * cast (F32) or split into FP16 hi/lo tiles (SPLIT16).  Replaces
 * SphericalHarmonicTransform.__post_init__/_build_tables
 * (src/arwen_global/spectral/transform.py:753-899) and GaussianGrid.create
 * (src/arwen_global/spectral/grid.py:97-126).  nlat/nlon are taken as given
 * (the Python layer applies the reference's shape rule, grid.py:26-94).
 * flags: SHT_FLAG_GEOMETRY_ONLY computes only the Gauss nodes and weights
 * (sht_plan_geometry works; transform calls fail); SHT_FLAG_GENERIC_FFT
 * selects the generic FFT kernels. */
int sht_plan_create(int truncation, int nlat, int nlon, double radius_m,
                    int precision, int flags, sht_plan** out_plan);
int sht_plan_destroy(sht_plan* plan);

/* Grow the plan's scratch for calls of up to `planes` planes (optional; calls
 * grow it on demand, which allocates and is therefore not capturable). */
int sht_plan_reserve(sht_plan* plan, int64_t planes);

/* Copy the FP64 geometry to host arrays of nlat doubles (any may be NULL). */
int sht_plan_geometry(const sht_plan* plan, double* mu, double* weights, double* coslat);

/* The plan's Legendre tables.  BASIS is P_nm, DBASIS dP_nm/dphi, ANALYSIS the
 * Gram-corrected 2 pi w P_nm rows, ROTATION (2 pi w / (a cos phi)) P_nm and
 * SHEAR (2 pi w / a) dP_nm/dphi (the vector analysis's weighted tables). */
#define SHT_TABLE_BASIS 0
#define SHT_TABLE_DBASIS 1
#define SHT_TABLE_ANALYSIS 2
#define SHT_TABLE_ROTATION 3
#define SHT_TABLE_SHEAR 4

/* Resident device bytes of one table: the equator-folded table in the plan's
 * element type plus, on a SPLIT16 plan, its FP16 hi/lo tile image and column
 * scales.  The reference's legendre_table_nbytes
 * (src/arwen_global/spectral/transform.py:936-954) reports the same per-table
 * figure for its banded tables. */
int sht_plan_table_bytes(const sht_plan* plan, int table, int64_t* bytes);

/* One table copied to host memory in the reference's dense layout, in the
 * plan's element type (double for F64, float for F32 and SPLIT16): BASIS and
 * DBASIS as [m][n][j] ((T+1) x (T+1) x nlat), ANALYSIS, ROTATION and SHEAR as
 * [m][j][n] ((T+1) x nlat x (T+1)), latitude row 0 southernmost, zero above
 * the triangle (n < m).  The northern rows are the folded table's southern
 * rows times the degree-parity sign (-1)^(n-m) (negated for DBASIS and SHEAR,
 * odd in latitude).  Replaces BandedLegendreTable.dense()
 * (src/arwen_global/spectral/transform.py:214-216), which the reference's
 * tests compare with its dense tables.  Synchronous; for tests and
 * inspection, not for a hot path. */
int sht_plan_read_table(const sht_plan* plan, int table, void* host_out);

/* Read and clear the plan's device error word (synchronises the plan's last
 * stream).  Returns SHT_ERR_DEVICE with a message if a kernel gave up on a
 * bounded wait. */
int sht_plan_check(sht_plan* plan);

/* Kernel kinds of the per-kernel timing counters. */
#define SHT_KIND_FFT_FORWARD 0   /* grid -> folded waist */
#define SHT_KIND_FFT_INVERSE 1   /* folded waist -> grid */
#define SHT_KIND_LEGENDRE_ANALYSIS 2
#define SHT_KIND_LEGENDRE_SYNTHESIS 3
#define SHT_KIND_PACK 4          /* spectral -> synthesis operand */
#define SHT_KIND_UNPACK 5        /* analysis output -> spectral */
#define SHT_KIND_ELEMENTWISE 6   /* project / Laplacian */
#define SHT_KIND_HELMHOLTZ 7
#define SHT_KIND_COUNT 8

/* Per-kernel device timing, the engine's counterpart of the reference's
 * StepProfiler (src/arwen_global/profile.py:1-50): when enabled, every kernel
 * launch of the plan is bracketed by CUDA events on its stream.  Launch
 * counters run always.  Not for use while a stream is being captured. */
int sht_plan_set_timing(sht_plan* plan, int enable);

/* Accumulated device milliseconds, launches and timed launches per kind
 * (arrays of n <= SHT_KIND_COUNT entries, any may be NULL); synchronises on
 * the recorded events; reset != 0 clears the counters. */
int sht_plan_read_timing(sht_plan* plan, double* ms, int64_t* launches, int64_t* timed,
                         int n, int reset);

/* Measured FP32 FFMA rate of the current device in TFLOP/s: register-only
 * fmaf chains on two 512-thread CTAs per SM, timed with CUDA events on
 * `stream` after a warm-up launch (about 10 ms of GPU time; synchronises on
 * the stream).  The denominator of the plain FP32 contraction's roofline.
 * A measurement helper of this engine; the reference has no counterpart
 * (its profiler, src/arwen_global/profile.py, times whole steps only). */
int sht_measure_fp32_peak(void* stream, double* tflops);

/* grid -> spectral.  SphericalHarmonicTransform.forward (transform.py:1486). */
int sht_forward(sht_plan* plan, const void* grid, int64_t planes, void* coeff, void* stream);

/* Size of the device buffer compiled into the library for
 * sht_forward_static_scratch (32 MiB, held on every GPU that loads it). */
#define SHT_STATIC_SCRATCH_BYTES (32u << 20)

/* grid -> spectral, like sht_forward, for callers that cannot allocate device
 * memory when they transform (a host callback, an allocator hook, a process
 * whose device budget belongs to an external memory manager).  It has no
 * counterpart in the reference.  Its scratch is the fixed
 * SHT_STATIC_SCRATCH_BYTES buffer above instead of the plan's on-demand
 * scratch, and it allocates nothing; a call that needs more (too many
 * planes) is rejected with SHT_ERR_ARG and the per-call plane limit in the
 * message.  FP32 and FP64 plans only.  The first call on a device looks the
 * buffer's address up (make it before any stream capture) and caches it per
 * device ordinal for the life of the process, so the cache assumes one
 * primary context per device: after cudaDeviceReset the cached address is
 * stale and the call must not be used again in that process.  Every call
 * shares the buffer, so calls that overlap on the GPU race on it. */
int sht_forward_static_scratch(sht_plan* plan, const void* grid, int64_t planes, void* coeff,
                               void* stream);

/* spectral -> grid.  SphericalHarmonicTransform.inverse (transform.py:1742). */
int sht_inverse(sht_plan* plan, const void* coeff, int64_t planes, void* grid, void* stream);

/* Host-resident fields.  The reference accepts host (numpy) arrays and
 * moves them to its backend's device inside forward/inverse
 * (transform.py:1486, 1742); these are that path for whole batches: planes
 * move host -> device -> host in chunks of `chunk` planes on three internal
 * streams, so the copies of neighbouring chunks overlap each other and the
 * transforms.  chunk = 0 selects the library's schedule: chunks of about a
 * sixteenth of the planes (even), ramped 2, 4, 8, ... planes at both ends of
 * the batch so the pipeline fills and drains in a few planes' copies.  Host buffers
 * should be page-locked (cudaHostAlloc / cudaHostRegister) for the copies to
 * run asynchronously; pageable memory works, without the overlap.  The
 * calls return when the output is on the host.  sht_round_trip_host is the
 * forward transform followed by the inverse (grid in, grid out, the
 * spectral coefficients never leave the device). */
int sht_forward_host(sht_plan* plan, const void* host_grid, int64_t planes, void* host_coeff,
                     int64_t chunk);
int sht_inverse_host(sht_plan* plan, const void* host_coeff, int64_t planes, void* host_grid,
                     int64_t chunk);
int sht_round_trip_host(sht_plan* plan, const void* host_grid, int64_t planes, void* host_out,
                        int64_t chunk);

/* d/dphi synthesis.  inverse_meridional_derivative (transform.py:1748). */
int sht_inverse_meridional_derivative(sht_plan* plan, const void* coeff, int64_t planes,
                                      void* grid, void* stream);

/* d/dlambda synthesis.  inverse_zonal_derivative (transform.py:1752). */
int sht_inverse_zonal_derivative(sht_plan* plan, const void* coeff, int64_t planes,
                                 void* grid, void* stream);

/* (east, north) physical gradient per metre.  gradient (transform.py:1762). */
int sht_gradient(sht_plan* plan, const void* coeff, int64_t planes, void* east,
                 void* north, void* stream);

/* vorticity/divergence -> (u, v).
 * VorticityDivergenceOperator.wind_from_vordiv (src/arwen_global/spectral/vector.py:36-52). */
int sht_wind_from_vordiv(sht_plan* plan, const void* vorticity, const void* divergence,
                         int64_t planes, void* u, void* v, void* stream);

/* (u, v) -> vorticity/divergence by integration by parts.
 * VorticityDivergenceOperator.vordiv_from_wind (vector.py:54-73). */
int sht_vordiv_from_wind(sht_plan* plan, const void* u, const void* v, int64_t planes,
                         void* vorticity, void* divergence, void* stream);

/* Vorticity/divergence from the Fourier waist of a stacked (u, v) pair,
 * `waist` = (2, planes, nlat, T+1) complex in the layout of
 * sht_fourier_waist (u first): the contraction half of vordiv_from_wind,
 * for a waist a band pipeline filled.
 * VorticityDivergenceOperator.vordiv_from_wind_waist / _vordiv_from_fourier
 * (vector.py:75-82, 113-134). */
int sht_vordiv_from_waist(sht_plan* plan, const void* waist, int64_t planes, void* vorticity,
                          void* divergence, void* stream);

/* The divergence alone from the same stacked (u, v) waist:
 * D = i m rot[u] - shear[v], each contraction over one field's rows.
 * VorticityDivergenceOperator.divergence_from_fourier (vector.py:136-166). */
int sht_divergence_from_waist(sht_plan* plan, const void* waist, int64_t planes,
                              void* divergence, void* stream);

/* Triangle mask and Imag(c[n,0]) = 0.  project (transform.py:1124-1144).
 * in and out may alias. */
int sht_project(sht_plan* plan, const void* in, int64_t planes, void* out, void* stream);

/* Multiply by -n(n+1)/a^2.  laplacian (transform.py:1798). */
int sht_laplacian(sht_plan* plan, const void* in, int64_t planes, void* out, void* stream);

/* Divide by -n(n+1)/a^2, zero degree 0, project.  inverse_laplacian (transform.py:1804). */
int sht_inverse_laplacian(sht_plan* plan, const void* in, int64_t planes, void* out,
                          void* stream);

/* Semi-implicit stage solve (I - tau_w L) y = r per total degree in the
 * vertical-mode basis.  VerticalModeSemiImplicit.solve_shifted
 * (src/arwen_global/semi_implicit.py:921-953) with helmholtz_inverse
 * (semi_implicit.py:585-609) applied as V diag(1/(1 + tau_w^2 k_n^2 lambda_j)) V^-1.
 * Host matrices (row-major float64): b (nlev x nlev+1), c (nlev+1 x nlev),
 * eigvec V (nlev x nlev), eigvec_inv V^-1 (nlev x nlev), eigenvalues (nlev).
 * Device arrays in the plan's complex type: divergence/theta (nlev, T+1, T+1),
 * lnps (T+1, T+1); results go to the out_* arrays (which may alias the inputs).
 * Degree zero passes through; outputs are projected. */
int sht_helmholtz_solve(sht_plan* plan, int nlev, const double* b, const double* c,
                        const double* eigvec, const double* eigvec_inv,
                        const double* eigenvalues, double tau_w,
                        const void* divergence, const void* theta, const void* lnps,
                        void* out_divergence, void* out_theta, void* out_lnps,
                        void* stream);

/* The same solve with the vertical operator kept on the device.  The
 * reference builds its VerticalStructureOperator once per run and its
 * per-(dt, alpha) inverse once per stage weight (semi_implicit.py:585-609,
 * 887-919); sht_vertical_create uploads B, C, V, V^-1 and the eigenvalues
 * (same host layout as sht_helmholtz_solve) once, in the plan's arithmetic
 * type.  sht_helmholtz_apply then does no allocation, no host copy and no
 * synchronisation, so it can be recorded in a CUDA graph.  An operator
 * serves plans of the same device and precision as the one it was created
 * with. */
int sht_vertical_create(sht_plan* plan, int nlev, const double* b, const double* c,
                        const double* eigvec, const double* eigvec_inv,
                        const double* eigenvalues, sht_vertical** out);
int sht_vertical_destroy(sht_vertical* op);
int sht_helmholtz_apply(sht_plan* plan, const sht_vertical* op, double tau_w,
                        const void* divergence, const void* theta, const void* lnps,
                        void* out_divergence, void* out_theta, void* out_lnps, void* stream);

/* An operator that also carries the modes of the thermodynamic block C B
 * (x_eigvec W, its inverse, and x_eigenvalues mu, (nlev+1) x (nlev+1) and
 * nlev+1, row-major; VerticalStructureOperator._build,
 * semi_implicit.py:551-577), which half_apply needs. */
int sht_vertical_create_modes(sht_plan* plan, int nlev, const double* b, const double* c,
                              const double* eigvec, const double* eigvec_inv,
                              const double* eigenvalues, const double* x_eigvec,
                              const double* x_eigvec_inv, const double* x_eigenvalues,
                              sht_vertical** out);

/* The three maps of VerticalModeSemiImplicit on (D, theta, ln ps), with
 * dt_w = dt (or tau) times the divergence weight:
 *   SHT_SEMI_SOLVE_SHIFTED  the IMEX stage solve (I - tau w L) y = r
 *                           (solve_shifted, semi_implicit.py:921-953; alpha ignored);
 *   SHT_SEMI_APPLY          the off-centred Crank-Nicolson step with weight
 *                           alpha (apply, semi_implicit.py:887-919);
 *   SHT_SEMI_HALF_APPLY     its square root (half_apply, semi_implicit.py:845-877;
 *                           needs sht_vertical_create_modes);
 *   SHT_SEMI_LINEAR_TENDENCIES  the weighted linear operator itself, dt_w = w:
 *                           D_t = w k^2 (B x), x_t = w (C D)
 *                           (linear_tendencies, semi_implicit.py:796-813; alpha
 *                           ignored, no degree-zero pass-through, metric 0).
 * Degree zero passes through and the outputs are projected (_finish,
 * semi_implicit.py:815-843).  The largest |D' - D| of the call is kept on
 * the device in the operator; sht_semi_implicit_metric reads it
 * (synchronising `stream`). */
#define SHT_SEMI_SOLVE_SHIFTED 0
#define SHT_SEMI_APPLY 1
#define SHT_SEMI_HALF_APPLY 2
#define SHT_SEMI_LINEAR_TENDENCIES 3
int sht_semi_implicit_map(sht_plan* plan, const sht_vertical* op, int mode, double dt_w,
                          double alpha, const void* divergence, const void* theta,
                          const void* lnps, void* out_divergence, void* out_theta,
                          void* out_lnps, void* stream);
int sht_semi_implicit_metric(const sht_vertical* op, double* max_divergence_increment,
                             void* stream);

/* solve_shifted fused with the synthesis of the solved divergence: the
 * solve writes D' straight into the folded synthesis operand, then the
 * Legendre synthesis and inverse FFT give divergence_grid
 * (nlev, nlat, nlon).  Equal to sht_helmholtz_apply followed by
 * sht_inverse of out_divergence, without the pack pass between them. */
int sht_helmholtz_synthesis(sht_plan* plan, const sht_vertical* op, double tau_w,
                            const void* divergence, const void* theta, const void* lnps,
                            void* out_divergence, void* out_theta, void* out_lnps,
                            void* divergence_grid, void* stream);

/* Autotuner settings of a plan (no counterpart call in the reference, whose
 * tile shapes and band splits are fixed in code; b200sht/autotune.py times
 * the combinations on the caller's plane count and keeps the fastest):
 *   SHT_TUNE_CONTRACTION 0: the plan's own contraction; 1: FP32 SIMT on a
 *                        split16 plan
 *   SHT_TUNE_FFT         0: register-resident FFT (where the grid allows);
 *                        1: shared-memory Stockham FFT
 *   SHT_TUNE_TILE_ORDER  tensor-core work order among equal-cost tiles:
 *                        0: row blocks of a column tile adjacent;
 *                        1: column tiles of a row block adjacent
 *   SHT_TUNE_TC_CTAS     tensor-core CTAs per launch; 0: one per SM
 *   SHT_TUNE_ACCUMULATORS tensor-core accumulators: 0: the main product in
 *                        three K-segment accumulators (split error ~3.6e-7 at
 *                        T511); 1: one, double-buffered so the epilogue
 *                        overlaps the next tile (~3 % faster pair, error
 *                        ~1.2e-6, still within 2e-6); 2: two K segments with
 *                        the data operand held in tensor memory (~1 % faster,
 *                        error ~6e-7)
 *   SHT_TUNE_SIMT_TILE   FP32 SIMT contraction tile shape (columns x rows):
 *                        0: 128 x 128; 1: 64 x 128 (less padding on the
 *                        ragged analysis blocks, more table loads); FP64
 *                        plans have the one shape 64 x 64
 * Set between calls, not while a call of the plan is in flight. */
#define SHT_TUNE_CONTRACTION 0
#define SHT_TUNE_FFT 1
#define SHT_TUNE_TILE_ORDER 2
#define SHT_TUNE_TC_CTAS 3
#define SHT_TUNE_ACCUMULATORS 4
#define SHT_TUNE_SIMT_TILE 5
int sht_plan_set_tuning(sht_plan* plan, int key, int value);
int sht_plan_get_tuning(sht_plan* plan, int key, int* value);

/* The Fourier waist in the reference's layout: (planes, nlat, T+1) complex,
 * the zonal spectrum of each grid row divided by nlon and cut at m = T
 * (FourierWaist, src/arwen_global/spectral/transform.py:417-629).  The
 * four calls are the two halves of the transform pair the reference names
 * so that band pipelines can fill and drain grid space a latitude band at
 * a time:
 *   sht_fourier_waist     grid -> waist                (fourier_waist, transform.py:1294-1404)
 *   sht_contract_waist    waist -> coefficients        (contract_waist / contract_values, 1435-1473)
 *   sht_contract_to_waist coefficients -> waist        (contract_to_waist, 1629-1650), with the
 *                         basis, the d/dphi basis, or the basis times i m
 *                         (gradient_waists' zonal half, 1770-1786)
 *   sht_waist_to_grid     waist -> grid                (waist_to_grid / waist_band_to_grid, 1704-1735)
 * sht_contract_waist(sht_fourier_waist(g)) is sht_forward(g) and
 * sht_waist_to_grid(sht_contract_to_waist(c, SHT_WAIST_BASIS)) is
 * sht_inverse(c), up to the rounding of the layout conversion. */
#define SHT_WAIST_BASIS 0
#define SHT_WAIST_DBASIS 1
#define SHT_WAIST_ZONAL 2
int sht_fourier_waist(sht_plan* plan, const void* grid, int64_t planes, void* waist,
                      void* stream);
int sht_contract_waist(sht_plan* plan, const void* waist, int64_t planes, void* coeff,
                       void* stream);
int sht_contract_to_waist(sht_plan* plan, const void* coeff, int64_t planes, int table,
                          void* waist, void* stream);
int sht_waist_to_grid(sht_plan* plan, const void* waist, int64_t planes, void* grid,
                      void* stream);

/* Batches: up to 4 plans (for instance 32 ensemble members at T126 as one
 * plan of 32 x 200 planes, and the T255 control as another) transformed as
 * one call.  The reference runs each member and truncation through its own
 * transform object (src/arwen_global/spectral/transform.py:1435-1490 and
 * 1629-1746 per call); here the Legendre contractions of all plans run in
 * ONE launch per direction: on SHT_PREC_SPLIT16 plans the persistent
 * tensor-core kernel walks the merged work list of every plan sorted by the
 * triangular per-order cost; F32/F64 plans run one SIMT launch per plan.
 * The FFT, pack and unpack launches stay per plan.  planes[i] is the plane
 * count of plan i (fixed for the batch); the arrays of plan i are laid out
 * as in sht_forward / sht_inverse.  The plans must be distinct, share one
 * device and one precision, and outlive the batch; a plan must not be used
 * by another call while a batch call that holds it is in flight. */
int sht_batch_create(int nplans, sht_plan* const* plans, const int64_t* planes,
                     sht_batch** out);
int sht_batch_destroy(sht_batch* batch);
int sht_batch_forward(sht_batch* batch, const void* const* grids, void* const* coeffs,
                      void* stream);
int sht_batch_inverse(sht_batch* batch, const void* const* coeffs, void* const* grids,
                      void* stream);

/* Semi-Lagrangian interpolation at departure points (the reference's
 * semilag/interpolate.py gather_batch / gather_linear_batch and the kernels
 * they launch, semilag/kernels.cu sl_gather_*, sl_gather5_*, sl_linear_*).
 *
 * sht_sl_tables_create builds the grid's geometry once (the reference's
 * SphericalGridTables.create, semilag/tables.py:136-258): the pole-extended
 * latitude tables of the four-point (and, for nlat >= 6, six-point)
 * meridional stencils, the row offsets and zonal shifts each extended row
 * reads, the reciprocal Lagrange denominators and the bracket lookup, in
 * float64 on the host and uploaded in the precision's element type
 * (SHT_PREC_F64: double, SHT_PREC_F32: float).  lat_rad: nlat ascending
 * Gauss latitudes; lon_rad (optional): checked to be i*2*pi/nlon.
 *
 * sht_sl_gather reads `fields` source volumes src[f][nlev][nlat][nlon] at the
 * departure coordinates xi (continuous zonal index), phi (latitude) and level
 * (continuous full-level index), each [nlev][nlat][nlon], into
 * out[f][nlev][nlat][nlon]: order 4 = tricubic, 6 = quintic horizontal with
 * the cubic vertical; limiter SHT_SL_QUASI_MONOTONE clips to the 2x2x2 cell
 * around the point; with deficit != 0 (cubic, limited) cut[f] receives raw
 * minus kept.  sht_sl_gather_linear is the trilinear value inside that cell.
 * Stream-ordered; every pointer is device memory the caller owns. */
typedef struct sht_sl_tables sht_sl_tables;
#define SHT_SL_NONE 0
#define SHT_SL_QUASI_MONOTONE 1
int sht_sl_tables_create(int nlat, int nlon, const double* lat_rad, const double* lon_rad,
                         int precision, sht_sl_tables** out);
int sht_sl_tables_destroy(sht_sl_tables* tables);
/* Latitude-band windows (the reference's semilag/tables.py BandWindow):
 * arrival rows [a0, a1) of a step read from fields that hold only rows
 * [s0, s1), the band and a row halo.  sht_sl_gather_band and
 * sht_sl_departure_band take coordinates / outputs / extrapolated wind of
 * the a1 - a0 arrival rows and sources / advecting wind of the s1 - s0 held
 * rows; brackets and weights are the whole grid's, so the values equal the
 * whole-grid calls' on those rows.  A read of a row outside the held rows
 * raises the window's escape flag (and reads the first held row instead);
 * sht_sl_window_escape reads it (synchronising `stream`) and/or clears it.
 * Buffer shapes of the band calls (nothing in the C layer can check them):
 * src (fields, nlev, s1 - s0, nlon); vx, vy, vz, level_rate (nlev, s1 - s0,
 * nlon); xi, phi, level, out, cut, the *_ex winds, move_m and move_k
 * (.., nlev, a1 - a0, nlon).
 * A window borrows `tables` (it keeps the pointer and reads the tables on
 * every band call): destroy every window of a tables object before
 * sht_sl_tables_destroy.  A window holds one escape flag, so the band calls
 * of one window are serialised on one stream; calls on different streams
 * would set and clear each other's flag. */
typedef struct sht_sl_window sht_sl_window;
int sht_sl_window_create(const sht_sl_tables* tables, int s0, int s1, int a0, int a1,
                         sht_sl_window** out);
int sht_sl_window_destroy(sht_sl_window* window);
int sht_sl_window_escape(sht_sl_window* window, int clear, int* escaped, void* stream);
int sht_sl_gather_band(const sht_sl_window* window, int order, int limiter, int deficit,
                       const void* src, int64_t fields, int nlev, const void* xi,
                       const void* phi, const void* level, void* out, void* cut, void* stream);
/* `solver`: 0 the fixed-point search, 1 Newton, 2 line-search Newton (the
 * three whole-grid calls below). */
int sht_sl_departure_band(const sht_sl_window* window, int solver, int nlev, const void* vx,
                          const void* vy, const void* vz, const void* level_rate,
                          const void* vx_ex, const void* vy_ex, const void* vz_ex,
                          const void* level_rate_ex, int iterations, double dt, double radius,
                          void* xi, void* phi, void* level, void* move_m, void* move_k,
                          void* stream);
/* Host copies of one width's tables (order 4 or 6): lat_ext[rows],
 * mrden[(nlat + 1) * order], mlut[bins], rowoff[rows], rowshift[rows];
 * any pointer may be null. */
int sht_sl_tables_read(const sht_sl_tables* tables, int order, double* lat_ext, double* mrden,
                       int32_t* mlut, int32_t* rowoff, int32_t* rowshift, int* rows, int* bins,
                       double* lut_scale);
int sht_sl_gather(const sht_sl_tables* tables, int order, int limiter, int deficit,
                  const void* src, int64_t fields, int nlev, const void* xi, const void* phi,
                  const void* level, void* out, void* cut, void* stream);
int sht_sl_gather_linear(const sht_sl_tables* tables, const void* src, int64_t fields, int nlev,
                         const void* xi, const void* phi, const void* level, void* out,
                         void* stream);
/* The fixed-point departure-point search (the reference's
 * semilag/trajectory.py departure_points with solver "fixed_point", kernels.cu
 * sl_departure_*): vx, vy, vz (geocentric Cartesian wind, m/s) and
 * level_rate (levels/s) at full levels, [nlev][nlat][nlon]; the *_ex fields
 * (the extrapolated flow) are read at the arrival points only.  All
 * `iterations` (>= 1) in one launch; writes the departure coordinates xi
 * (continuous zonal index), phi (radians), level (continuous level index,
 * clamped to [-1/2, nlev - 1/2]) and the last iteration's move in metres
 * and in levels.  radius: the sphere's radius in metres. */
int sht_sl_departure(const sht_sl_tables* tables, int nlev, const void* vx, const void* vy,
                     const void* vz, const void* level_rate, const void* vx_ex,
                     const void* vy_ex, const void* vz_ex, const void* level_rate_ex,
                     int iterations, double dt, double radius, void* xi, void* phi,
                     void* level, void* move_m, void* move_k, void* stream);
/* The same search solved by Newton's method (the reference's opt-in
 * "newton" solver of trajectory.departure_points): per iteration the
 * residual of the fixed-point map in the local east / north / level frame
 * and the trilinear interpolant's Jacobian, (I - M) d = r solved directly,
 * the plain step where the system is near-singular, at a pole, or the
 * residual stopped shrinking.  Same arguments and fixed point as
 * sht_sl_departure. */
int sht_sl_departure_newton(const sht_sl_tables* tables, int nlev, const void* vx,
                            const void* vy, const void* vz, const void* level_rate,
                            const void* vx_ex, const void* vy_ex, const void* vz_ex,
                            const void* level_rate_ex, int iterations, double dt, double radius,
                            void* xi, void* phi, void* level, void* move_m, void* move_k,
                            void* stream);
/* The line-search Newton search (the reference's opt-in "newton_ls" solver,
 * kernels.cu sl_departure_newton_ls_*): the Newton direction (or the
 * residual where the 3 x 3 system is near-singular or at a pole), capped at
 * 20 residuals and halved at most four times until the residual in grid
 * cells falls by the Armijo factor 1 - 1e-4 alpha; a point whose residual is
 * below 1e-4 cells stops.  move_m / move_k report the step at the returned
 * point (its linearised distance to the root), not the last move.  Same
 * arguments and fixed point as sht_sl_departure. */
int sht_sl_departure_newton_ls(const sht_sl_tables* tables, int nlev, const void* vx,
                               const void* vy, const void* vz, const void* level_rate,
                               const void* vx_ex, const void* vy_ex, const void* vz_ex,
                               const void* level_rate_ex, int iterations, double dt,
                               double radius, void* xi, void* phi, void* level, void* move_m,
                               void* move_k, void* stream);

/* The flow deformation the trajectory must stay inside (the reference's
 * semilag/trajectory.py lipschitz, 1174-1420): at every point of the arrival
 * rows [a0, a1), the Jacobian of (vx, vy, vz, level_rate) -- zonal centred
 * differences, the three-point formula on the Gauss latitudes with the pole
 * row read half a turn round beyond a pole, centred level differences with
 * one-sided ends -- projected on the local east/north basis; out
 *   maxima[5]  = max over the points of the spectral norm of the mixed-unit
 *                3 x 3 (vertical entries scaled by reference_length), its
 *                Frobenius norm, the spectral norm of the horizontal 2 x 2,
 *                |d(level rate)/dk| and the spectral norm of the balanced
 *                3 x 3 (per second);
 *   minima[2]  = min det(I + (dt/2) J) (departure side, the wind) and
 *                min det(I - (dt/2) J_ex) (arrival side, the extrapolated
 *                wind, or the wind when vx_ex is NULL);
 *   argmin[2]  = where each minimum sits, flat (level, arrival row, lon),
 *                the first in that order among equal values.
 * The wind holds rows [held0, held0 + held_rows) of the grid, the
 * extrapolated wind [ex_held0, ex_held0 + ex_held_rows); both must hold the
 * arrival rows and one row either side (the pole row at a pole), else
 * SHT_ERR_ARG (a halo escape).  nlev >= 2.  Synchronises `stream`.  The
 * tables' element type is the arrays'.  The call's scratch (per-CTA
 * partials, row and column tables) belongs to the tables object: one call
 * at a time per tables object. */
int sht_sl_lipschitz(const sht_sl_tables* tables, int nlev, int a0, int a1, const void* vx,
                     const void* vy, const void* vz, const void* level_rate, int held0,
                     int held_rows, const void* vx_ex, const void* vy_ex, const void* vz_ex,
                     const void* level_rate_ex, int ex_held0, int ex_held_rows, double dt,
                     double radius, double reference_length, double* maxima, double* minima,
                     int64_t* argmin, void* stream);

/* Fused right-hand-side kernels of the dycore step (the reference's
 * spectral/fused.py momentum_bernoulli_kernel, tracer_flux_kernel,
 * scalar_tendency_kernel, vertical_flux_divergence_kernel and their numpy
 * specifications in dynamics.py).  precision: SHT_PREC_F64 (double) or
 * SHT_PREC_F32 (float).  Volumes are C-order (nlev, nlat, nlon), horiz =
 * nlat * nlon; `blocks` counts leading (tracer) blocks of the scalar-side
 * arrays, the other operands being one shared block.
 *   momentum_bernoulli: coriolis, grad_lnps_east/north are (nlat, nlon),
 *     broadcast over levels; mu = (zeta + f) v - wu - R Tv pg ge,
 *     mv = -(zeta + f) u - wv - R Tv pg gn, bern = (u^2 + v^2)/2 + phi.
 *   tracer_flux: flux_east = (dp s) u, flux_north = (dp s) v.
 *   scalar_tendency: out = (-horizontal - vertical - s dp_t) / dp.
 *   vertical_flux_divergence: omega_half and p_half (nlev + 1, nlat, nlon),
 *     p_full (nlev, ...); the van Leer limited upstream flux through every
 *     interface (zero at the top and bottom), out[k] = F[k+1] - F[k]. */
int sht_rhs_momentum_bernoulli(int precision, int64_t nlev, int64_t horiz, const void* zeta,
                               const void* coriolis, const void* u, const void* v, const void* wu,
                               const void* wv, const void* tv, const void* pg,
                               const void* grad_lnps_east, const void* grad_lnps_north,
                               const void* geopotential, double gas_constant, void* mu, void* mv,
                               void* bernoulli, void* stream);
int sht_rhs_tracer_flux(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                        const void* dp, const void* scalar, const void* u, const void* v,
                        void* flux_east, void* flux_north, void* stream);
int sht_rhs_scalar_tendency(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                            const void* horizontal, const void* vertical, const void* scalar,
                            const void* dp_t, const void* dp, void* out, void* stream);
int sht_rhs_vertical_flux_divergence(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                                     const void* scalar, const void* omega_half,
                                     const void* p_full, const void* p_half, void* out,
                                     void* stream);

/* Spectral fields at arbitrary points (the reference's spectral/sampling.py
 * sample_scalar / sample_gradient; sample_wind is the gradient of the
 * inverse Laplacians).  sht_sampler_create builds the x-independent
 * recurrence factors of truncation T once.  sht_sample: coeff_mn is
 * complex128 [fields][m][n] (the [n, m] coefficients transposed), lat/lon
 * in radians [npoints]; gradient == 0: out0[fields][npoints] = the field;
 * gradient != 0: out0 = eastward, out1 = northward gradient (physical,
 * 1 / (radius cos phi) and 1 / radius applied; points off the poles).
 * FP64 throughout, device pointers. */
typedef struct sht_sampler sht_sampler;
int sht_sampler_create(int truncation, sht_sampler** out);
int sht_sampler_destroy(sht_sampler* sampler);
int sht_sample(sht_sampler* sampler, const void* coeff_mn, int64_t fields, int64_t npoints,
               const double* lat_rad, const double* lon_rad, int gradient, double radius,
               double* out0, double* out1, void* stream);
/* The packed real basis blocks of the reference's device sampler
 * (spectral/sampling.py packed_basis, 198-237) at npoints points (device
 * lat/lon in radians), each block [2 K][npoints], K = (T+1)(T+2)/2, rows in
 * the packed order of triangle_index (order-major, n fastest), in FP64 or
 * FP32 (out_precision SHT_PREC_F64 / SHT_PREC_F32).  gradient == 0: out0 =
 * [mult P cos(m lam); -mult P sin(m lam)], so that [Re c | Im c] @ out0 is
 * the field; gradient != 0: out0 = [-m mult P sin; -m mult P cos] (zonal),
 * out1 = [mult dP/dphi cos; -mult dP/dphi sin] (meridional); mult = 1 at
 * m = 0, 2 above.  The values are sht_sample's recurrence. */
int sht_sample_packed_basis(sht_sampler* sampler, int64_t npoints, const double* lat_rad,
                            const double* lon_rad, int gradient, int out_precision, void* out0,
                            void* out1, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B200SHT_H */
