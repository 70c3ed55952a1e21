/*
 * fastlpr_b200 -- C ABI of the B200 implementation of fastLPR's NUFFT path
 * (local polynomial regression with GCV, kernel density estimation with LCV).
 *
 * Conventions for every entry point:
 *   - returns int status: FLPR_OK (0) or a negative FLPR_ERR_* code;
 *     flpr_last_error() gives a message for the calling thread;
 *   - pointers named d_* are device pointers, h_* host pointers;
 *   - `stream` is a cudaStream_t passed as void*; work is only enqueued,
 *     the call does not synchronise unless its comment says so;
 *   - the library allocates no device memory: callers pass workspaces whose
 *     size they obtain from the matching *_ws query.
 *
 * Reference paths cited below are relative to fastLPR_py/src/fastlpr/.
 */
#ifndef FASTLPR_B200_H
#define FASTLPR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLPR_OK 0
#define FLPR_ERR_ARG (-1)         /* invalid argument or unsupported shape */
#define FLPR_ERR_CUDA (-2)        /* CUDA runtime error */
#define FLPR_ERR_CUFFT (-3)       /* cuFFT error */
#define FLPR_ERR_WORKSPACE (-4)   /* workspace smaller than the query said */
#define FLPR_ERR_TIMEOUT (-5)     /* a bounded device-side wait ran out */

#define FLPR_PREC_F32 0           /* FP32 grids/FFT/products, FP64 solve and reductions */
#define FLPR_PREC_F64 1           /* FP64 throughout */

#define FLPR_MAX_DIMS 3
#define FLPR_MAX_CHANNELS 64

typedef struct flpr_handle_s* flpr_handle_t;

const char* flpr_last_error(void);
int flpr_version(void);
/* Number of CUDA kernels launched by this library since it was loaded
 * (cuFFT's own kernels are not counted). */
int64_t flpr_launch_count(void);

/* Tuning parameters, process-wide (they hold for every later call on every
 * device; calls already enqueued keep the values they were launched with).
 * Set by the autotuner of the Python host (fastlpr_b200/autotune.py).
 *   FLPR_TUNE_SPREAD_ITEM_POINTS: points per spread work item (one CTA),
 *     256..65536, default 4096;
 *   FLPR_TUNE_FUSED_CHUNK_MB: column-pass output budget of the fused 2-D
 *     convolution (bandwidths per chunk), 8..16384 MB, default 768. */
#define FLPR_TUNE_SPREAD_ITEM_POINTS 0
#define FLPR_TUNE_FUSED_CHUNK_MB 1
#define FLPR_TUNE_COUNT 2
int flpr_set_tuning(int param, int value);
int flpr_get_tuning(int param);

/* Handle: owns cuFFT plans (without work areas) for one device. */
int flpr_create(flpr_handle_t* out, int device);
int flpr_destroy(flpr_handle_t handle);

/* ---------------------------------------------------------------------
 * (1) Point statistics.  Replaces the numpy reductions of model.py:58-68
 * (mean, std ddof=1, min, max per axis) and api.py:1025 (column sums).
 * d_x: (n, d) row-major float64.  d_stats receives 4*d doubles:
 * [min(d), max(d), mean(d), M2(d)] with M2 = sum (x - mean)^2.
 * --------------------------------------------------------------------- */
size_t flpr_point_stats_ws(int d, int64_t n);
int flpr_point_stats(int d, int64_t n, const double* d_x, double* d_stats,
                     void* d_ws, size_t ws_bytes, void* stream);

/* (1b) The same point statistics without any device allocation by the
 * caller or the library.  This entry point has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory at the
 * point where they need the statistics: code running under a host
 * application that owns every device buffer through its own pool (a
 * plugin or FFI caller that may not call cudaMalloc/cudaFree), or a caller
 * that must not trigger the implicit device synchronisation of an
 * allocation.  The caller still passes d_x and d_stats.
 * The per-block partial results go to a static device array inside the
 * library (1024 blocks x 8 axes x 40 bytes = 320 KiB, held by every GPU that
 * loads the library until the process exits).  Limits: d <= 8 (larger d is
 * rejected with FLPR_ERR_ARG and a message); any n.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress), so
 * make the first call on each device before any stream capture begins.
 * The address is cached per device context (its cuCtxGetId): after a
 * device reset, or under another context of the same device, the next call
 * looks it up again, so again call it once before capturing there.
 * All calls share the array: two calls whose kernels overlap on the GPU
 * (different streams, no ordering between them) race and may return wrong
 * statistics; calls on one stream are ordered and safe. */
int flpr_point_stats_noalloc(int d, int64_t n, const double* d_x, double* d_stats,
                             void* stream);

/* ---------------------------------------------------------------------
 * (2) Gaussian-gridding spread of every channel onto the periodic L^d grid
 * (NUFFT type-1 spreading).  Replaces fused_spreading_dispatch
 * (spreading_fused.py:310-332) and nufft_accumulate_cython
 * (_nufft_accel.pyx:32-76), including the knot mapping of
 * convolution.py:176-213 and scale_knots (nufftn_type1.py:140-176).
 *
 * h_kmap: per axis 9 doubles {mean, std, center, xs_min, xs_scale,
 *   knot_scale, knot_r0, knot_shift, hx}; the kernel applies
 *   xs = (x-mean)/std - center;  xn = (xs-xs_min)/xs_scale*knot_scale + r0;
 *   xn = mod(xn+0.5, 1) - 0.5;  k = mod((xn+shift)*2pi, 2pi);
 *   m = rint(k/hx); taps j in [-msp, msp], weight exp(-sum diff^2/(4 tau)).
 * Channels: if ones_channel, channel 0 is the constant 1; the remaining
 *   nchan-ones_channel channels are h_cols[i] (device float64 arrays of n).
 * d_grid_out: (nchan, L...) real, float (FLPR_PREC_F32) or double, scaled
 *   by 1/n (the 1/M of nufftn_type1.py:709-711).
 * Accumulation is per-tile in shared memory after binning the points by
 * tile; FLPR_PREC_F32 accumulates in 64-bit fixed point (order independent,
 * deterministic), FLPR_PREC_F64 in float64.
 * --------------------------------------------------------------------- */
size_t flpr_spread_ws(int d, int64_t n, const int* h_L, int msp, int nchan, int prec);
int flpr_spread(int d, int64_t n, const double* d_x, const double* h_kmap,
                const int* h_L, int msp, const double* h_tau,
                int nchan, int ones_channel, const double* const* h_cols,
                void* d_grid_out, int prec, void* d_ws, size_t ws_bytes, void* stream);
/* The same spread with the knot maps read on the device (d_kmap, d x 9, the
 * rows of h_kmap above; h_hx: the knot spacings of the axes), so that it can
 * be enqueued before the point statistics reach the host.  Same workspace
 * as flpr_spread.  No separate reference counterpart: it is the spread of
 * nufftn_type1.py:378-772 with the geometry of model.py:58-68 and
 * convolution.py:190-208 formed on the device. */
int flpr_spread_dkmap(int d, int64_t n, const double* d_x, const double* d_kmap,
                      const double* h_hx, const int* h_L, int msp, const double* h_tau,
                      int nchan, int ones_channel, const double* const* h_cols,
                      void* d_grid_out, int prec, void* d_ws, size_t ws_bytes, void* stream);
/* The FP64 grid of the last FLPR_PREC_F32 spread that used this
 * workspace with the same d, n, L, msp and nchan: the exact fixed-point sums
 * (before their rounding to FP32) times 1/n, as (nchan, L...) float64.  The
 * FP32 path evaluates bandwidths whose kernel covers few points with FP64
 * planes; this gives them their grids without a second spread.  No
 * reference counterpart (the reference spreads once, in one precision). */
int flpr_spread_grid64(int d, int64_t n, const int* h_L, int msp, int nchan, const void* d_ws,
                       size_t ws_bytes, double* d_grid64, void* stream);
/* The same for the first nout channels only, as (nout, L...) float64 (the
 * ones channel alone gives the FP64 moment planes of order-2 fits). */
int flpr_spread_grid64_channels(int d, int64_t n, const int* h_L, int msp, int nchan, int nout,
                                const void* d_ws, size_t ws_bytes, double* d_grid64,
                                void* stream);
/* Knot maps d_kmap (d x 9) from the point statistics d_stats (4 x d:
 * minimum, maximum, mean, M2 as flpr_point_stats writes them) and the
 * host-known per-axis constants of the grid (ks, r0: the knot range of
 * convolution.py:190-208; hx = 2 pi / L), in the operations and order of the
 * host geometry (model.py:58-68, nufftn_type1.py:164-166). */
int flpr_knot_map(int d, int64_t n, const double* d_stats, const double* h_ks,
                  const double* h_r0, const double* h_hx, double* d_kmap, void* stream);

/* ---------------------------------------------------------------------
 * (3) Forward FFT of the spread grids: real-to-complex over all axes,
 * batched over channels.  Replaces the fft/fftshift/ifftshift chain of
 * nufftn_type1.py:701-711 and convolution.py:235-236 (the shifts cancel).
 * d_spec: (nchan, L0, .., L_{d-1}/2+1) complex (float2 or double2).
 * --------------------------------------------------------------------- */
size_t flpr_forward_fft_ws(flpr_handle_t handle, int d, const int* h_L, int nchan, int prec);
int flpr_forward_fft(flpr_handle_t handle, int d, const int* h_L, int nchan,
                     void* d_grid, void* d_spec, int prec,
                     void* d_ws, size_t ws_bytes, void* stream);

/* (3b) Oversampled spreading (accuracy >= 7): nufftn_type1.py:693-770 and
 * the ifftshift of convolution.py:235-236.  d_in: (nchan, Lin.., Lin_last/2+1)
 * R2C spectra of the ratio*L grids from flpr_forward_fft; d_out receives
 * (nchan, Lout.., Lout_last/2+1): the central Lout frequencies of each axis,
 * divided by ratio^d and by the Gaussian spreading transform
 * sqrt(prod tau / pi^d) exp(-sum tau_a f_a^2), in standard frequency order. */
int flpr_oversample_crop(int d, const int* h_Lout, const int* h_Lin, int nchan,
                         const double* h_tau, int ratio, const void* d_in, void* d_out,
                         int prec, void* stream);

/* ---------------------------------------------------------------------
 * (4) Per-axis kernel-moment spectra.  The Gaussian kernel of
 * kernel.py:330-357 is separable, so the spectrum of K(u)*u^a on the padded
 * grid (convolution.py:318-794, design_matrix_optimized.py:216-436) is
 * (1/sqrt(2 pi)) * prod_d F[d][h][a_d].  This computes F for
 * a = 0..npow-1: the 1-D factor exp(-u^2/2) u^a / h_d sampled on
 * linspace(lo_d, hi_d, G_d), zero padded with floor((L-G)/2)+1 leading
 * zeros, FFT of length L_d.  d_F: per axis d, (H, npow, L_d) double2,
 * axes stacked.  d_sum0: (d, H) sums of the a=0 factor over the grid (used
 * for the "too small bandwidth" filter of convolution.py:542-605).
 * --------------------------------------------------------------------- */
size_t flpr_kernel_factors_ws(flpr_handle_t handle, int d, const int* h_L, int H, int npow);
int flpr_kernel_factors(flpr_handle_t handle, int d, const int* h_G, const int* h_L,
                        const double* h_lo, const double* h_hi, int H, const double* d_h,
                        int npow, void* d_F, double* d_sum0,
                        void* d_ws, size_t ws_bytes, void* stream);

/* ---------------------------------------------------------------------
 * (5) Spectral multiply + inverse FFT + crop for a list of products.
 * Product p multiplies channel chan[p] by the kernel spectrum of bandwidth
 * hidx[p] and per-axis exponents pow[p*d .. p*d+d-1], inverts, keeps the
 * real part and crops [qout0_d, qout0_d + G_d) per axis.  Replaces
 * nufft_convolve (convolution.py:904-951).  Output plane p goes to
 * d_out + p * prod(G) elements (float or double, per prec); when
 * add_eps is set the float64 machine epsilon is added (regression.py:116).
 * h_scale: global factor applied to every product (1/(sqrt(2pi) prod L)).
 * --------------------------------------------------------------------- */
size_t flpr_conv_ws(flpr_handle_t handle, int d, const int* h_L, int nprod, int prec);
int flpr_conv(flpr_handle_t handle, int d, const int* h_G, const int* h_L, const int* h_qout,
              int H, int npow, const void* d_spec, const void* d_F,
              int nprod, const int* h_chan, const int* h_hidx, const int* h_pow,
              double scale, int add_eps, void* d_out, int prec,
              void* d_ws, size_t ws_bytes, void* stream);

/* (5a) flpr_conv for d = 2 as two passes of 1-D transforms: per distinct
 * (channel, bandwidth, axis-0 exponent) the channel spectrum times the
 * axis-0 factor, inverse FFT along axis 0 and rows qout[0]..+G0-1 kept
 * (shared by every product with that triple); per product those rows times
 * the axis-1 factor and `scale`, C2R along axis 1 and columns
 * qout[1]..+G1-1 kept.  Same arguments (d = 2) and output as flpr_conv;
 * about half the transform work and a quarter of the traffic of the full
 * 2-D inverse per product. */
size_t flpr_conv2d_sep_ws(flpr_handle_t handle, const int* h_G, const int* h_L, int nprod,
                          int prec);
int flpr_conv2d_sep(flpr_handle_t handle, const int* h_G, const int* h_L, const int* h_qout,
                    int H, int npow, const void* d_spec, const void* d_F, int nprod,
                    const int* h_chan, const int* h_hidx, const int* h_pow, double scale,
                    int add_eps, void* d_out, int prec, void* d_ws, size_t ws_bytes,
                    void* stream);

/* (5b) Non-separable (radial) kernels: kernel.py:310-431 (epanechnikov,
 * tricube, quartic/biweight, triweight, uniform; also gaussian and
 * gaussian_ft) for compute_kernel_fourier (convolution.py:318-652) and
 * nufft_convolve (convolution.py:797-953).  A radial kernel of ||u|| does not
 * factor over the axes, so its moment planes K(u) prod_a u_a^p_a / prod_a h_a
 * (u = x / h on linspace(lo, hi, G) per axis, padded with floor((L-G)/2)+1
 * leading zeros) are sampled on the full L grid and transformed (D2Z).
 * kernel_id: 0 gaussian, 1 gaussian_ft, 2 epanechnikov, 3 tricube,
 * 4 quartic, 5 triweight, 6 uniform.  h_pow: (nelem, d) exponents.
 * d_K: (nelem, H, L0.., L_last/2+1) complex128, item e*H + h.
 * flpr_conv_full: flpr_conv with d_K in place of the per-axis factors;
 * product p multiplies channel h_chan[p] by kernel spectrum h_kidx[p]
 * (< nkern); same output, scale, eps and workspace (flpr_conv_ws). */
size_t flpr_kernel_spectra_ws(flpr_handle_t handle, int d, const int* h_L, int nitems);
int flpr_kernel_spectra(flpr_handle_t handle, int d, const int* h_G, const int* h_L,
                        const double* h_lo, const double* h_hi, int kernel_id, int H,
                        const double* d_h, int nelem, const int* h_pow, void* d_K, void* d_ws,
                        size_t ws_bytes, void* stream);
int flpr_conv_full(flpr_handle_t handle, int d, const int* h_G, const int* h_L, const int* h_qout,
                   int nkern, const void* d_spec, const void* d_K, int nprod, const int* h_chan,
                   const int* h_kidx, double scale, int add_eps, void* d_out, int prec,
                   void* d_ws, size_t ws_bytes, void* stream);

/* ---------------------------------------------------------------------
 * (6) Local polynomial solve at every grid point and bandwidth.
 * Replaces solve_regression_system (regression.py:162-277) and the
 * closed forms of lwp_formulas.py.  d_S: ns planes of (H, M) (M = prod G),
 * packed lower-triangular column-major; d_T: nt*C planes ordered [i][c] of
 * (HT, M) for the first HT <= H bandwidths.  Order 0:
 * m = t / max(s, max(s)*reg).  Order >= 1: lambda = 1e-6 * max |diag S|
 * over all points and all H bandwidths, m = e1' (S + lambda I)^-1 T by an
 * FP64 LDL' factorisation per (point, bandwidth) (partial-pivoting
 * elimination where a pivot vanishes).  d_m: (HT, M, C) float64.
 * d_scalar: one double of device scratch (receives lambda or max(s)).
 * --------------------------------------------------------------------- */
int flpr_solve(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
               const void* d_T, double reg, double* d_m, double* d_scalar, int prec,
               void* stream);

/* (6b) flpr_solve fused with the dual-form reductions: the same lambda
 * and solve, but m is written only for the first nkeep channels
 * (d_mkeep: (HT, M, nkeep)) and d_dots[c][h] = sum_g m_c(g) Q[g][c] is
 * accumulated for every channel c < C (C <= 32; d_dots (C, HT) overwritten)
 * with Q from flpr_deposit. */
int flpr_solve_reduce(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
                      const void* d_T, double reg, int nkeep, double* d_mkeep, const double* d_Q,
                      double* d_dots, double* d_scalar, int prec, void* stream);
/* (6b') The same with lambda (or max s) given in d_scalar instead of formed
 * from these planes: when the bandwidths of one sweep are split between an
 * FP64 group (kernels covering few points) and the FP32 group, the
 * reference's lambda over all bandwidths (regression.py:243-267) is the
 * larger of the two groups' (flpr_scalar_of). */
int flpr_solve_reduce_given(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
                            const void* d_T, double reg, int nkeep, double* d_mkeep,
                            const double* d_Q, double* d_dots, const double* d_scalar, int prec,
                            void* stream);
/* lambda (order >= 1) or max s (order 0) of the planes d_S (ns, H, M), as
 * flpr_solve forms it, raised to *d_floor when d_floor is not NULL. */
int flpr_scalar_of(int order, int nt, int H, int64_t M, const void* d_S, int prec,
                   const double* d_floor, double* d_scalar, void* stream);

/* (6c) Fused 2-D FP32 convolution + solve + dual-form reductions: the
 * whole inverse-transform / solve stage of a 2-D GCV sweep in one call,
 * replacing flpr_conv (S and T) + flpr_solve_reduce for FLPR_PREC_F32.
 * Separable kernel spectrum: a column pass (axis-0 factor, inverse FFT,
 * crop) shared by all moments with the same axis-0 exponent, then a row
 * pass (axis-1 factor, C2R, crop) fused with the FP64 solve; two real row
 * products share one complex transform.  Replaces nufft_convolve
 * (convolution.py:904-951) for S (regression.py:130-145) and T
 * (regression.py:802-817, 1516-1533) plus solve_regression_system.
 * d_spec: (1 + C, L0, L1/2+1) float2 from flpr_forward_fft (channel 0 = ones,
 * then C value channels of which the first ny are responses); d_F from
 * flpr_kernel_factors for these H bandwidths; d_Q (M, C) from flpr_deposit.
 * Outputs: d_S (ns, H, M) float (S planes), d_my (H, M, ny) fitted grids,
 * d_dots (C, H) = sum_g m_c(g) Q[g][c], d_scalar (lambda or max s).
 * Supported when flpr_lpr2d_fused_supported() returns 1: L0, L1 powers of
 * two in [64, 1024], C <= 32, order <= 2 (shared-memory limits). */
int flpr_lpr2d_fused_supported(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                               int C);
size_t flpr_lpr2d_fused_ws(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                           int C);
int flpr_lpr2d_fused(const int* h_G, const int* h_L, const int* h_qout, int H, int npow, int order,
                     int C, int ny, const void* d_spec, const void* d_F, double scale,
                     const double* d_Q, double reg, float* d_S, double* d_my, double* d_dots,
                     double* d_scalar, void* d_ws, size_t ws_bytes, void* stream);
/* The same with lambda raised to *d_scalar_floor (the other group's, see
 * flpr_solve_reduce_given) before the solves; d_scalar receives the
 * union's value. */
int flpr_lpr2d_fused_floor(const int* h_G, const int* h_L, const int* h_qout, int H, int npow,
                           int order, int C, int ny, const void* d_spec, const void* d_F,
                           double scale, const double* d_Q, double reg, float* d_S, double* d_my,
                           double* d_dots, double* d_scalar, const double* d_scalar_floor,
                           void* d_ws, size_t ws_bytes, void* stream);

/* The T pass of flpr_lpr2d_fused on FP64 S planes formed by the caller
 * (d_S64: (ns, H, M) float64, the moment matrices of every kept bandwidth
 * in FP64, e.g. from the exact FP64 grid of the ones channel) with lambda
 * (order >= 1) or max s (order 0) already in *d_scalar: the FP32 column and
 * row passes of the value channels, the per-point FP64 solves on the FP64
 * moment matrices and the dual-form reductions.  The local-quadratic
 * moment systems are then factorised from FP64 planes while the channels'
 * transforms stay FP32.  Same workspace as flpr_lpr2d_fused. */
int flpr_lpr2d_fused_t(const int* h_G, const int* h_L, const int* h_qout, int H, int npow,
                       int order, int C, int ny, const void* d_spec, const void* d_F, double scale,
                       const double* d_Q, double reg, const double* d_S64, const double* d_scalar,
                       double* d_my, double* d_dots, void* d_ws, size_t ws_bytes, void* stream);

/* The fused 2-D passes in either precision (prec FLPR_PREC_F32: float2
 * spectra and transforms; FLPR_PREC_F64: complex128 spectra, FP64
 * transforms, factor entries kept down to 1e-15 of their peak) and for a
 * chosen part (mode): 0 = S pass, lambda (floored by *d_scalar_floor when
 * given) and T pass, as flpr_lpr2d_fused_floor; 1 = the S planes only
 * (d_S: (ns, H, M) in prec; d_spec may then hold the ones channel alone);
 * 2 = the T pass on FP64 S planes d_S64 with lambda already in *d_scalar,
 * as flpr_lpr2d_fused_t.  Same outputs and workspace rules as
 * flpr_lpr2d_fused; the size query and support test take the precision. */
int flpr_lpr2d_fused_ex_supported(int prec, const int* h_G, const int* h_L, const int* h_qout,
                                  int H, int order, int C);
size_t flpr_lpr2d_fused_ex_ws(int prec, const int* h_G, const int* h_L, const int* h_qout, int H,
                              int order, int C);
int flpr_lpr2d_fused_ex(int prec, int mode, const int* h_G, const int* h_L, const int* h_qout,
                        int H, int npow, int order, int C, int ny, const void* d_spec,
                        const void* d_F, double scale, const double* d_Q, double reg, void* d_S,
                        const double* d_S64, double* d_my, double* d_dots, double* d_scalar,
                        const double* d_scalar_floor, void* d_ws, size_t ws_bytes, void* stream);

/* ---------------------------------------------------------------------
 * (7) Interpolation + GCV / Hutchinson reductions over the points.
 * Replaces the yhat interpolation and RSS of api.py:645-741 /
 * regression.py:280-471 and the probe interpolation and p'phat, p'p sums of
 * regression.py:1256-1300.  Multilinear clamped interpolation on the raw
 * grid (interp_optimized.py:60-130).  h_ax: per axis {x0, dx} with
 * dx = axis[1]-axis[0]; h_G grid sizes.  d_m: (H, M, C) float64 with
 * C = ny + R: the first ny channels are the response columns, the next R
 * the probes.  h_ycols: ny device float64 arrays (n); h_pcols: R arrays.
 * d_rss: (H, ny) sums of (y - yhat)^2; d_pdot: (R, H) sums of p*phat;
 * d_pp: (R) sums of p*p.  Outputs are overwritten.
 * --------------------------------------------------------------------- */
size_t flpr_interp_reduce_ws(int64_t n, int H, int ny, int R);
int flpr_interp_reduce(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G,
                       int H, int ny, int R, const double* d_m,
                       const double* const* h_ycols, const double* const* h_pcols,
                       double* d_rss, double* d_pdot, double* d_pp,
                       void* d_ws, size_t ws_bytes, void* stream);

/* (7b) Dual form of (7): the adjoint of the interpolation.
 * For channel values v_c (h_cols[c], c < C) at the raw points this deposits
 * Q[g][c] = sum_i w_ig v_ic (d_Q: (M, C)), the stencil weights of
 * sum_i interp(m)_i^2 (d_B: (M, P) with P = 2^d (2^d + 1) / 2 corner pairs per
 * base cell) and d_sq[c] = sum_i v_ic^2, so that
 *   sum_i v_ic interp(m)_i = sum_g m(g) Q[g][c]   and
 *   sum_i interp(m)_i^2    = sum_b sum_pairs B[b][p] m(b+c_k) m(b+c_k').
 * Same weights and clamping as flpr_interp_reduce (interp_optimized.py:60-130);
 * the RSS and p'phat of regression.py:1256-1300 and api.py:645-741 then cost
 * grid-domain dot products instead of one interpolation per point,
 * bandwidth and channel.  Outputs are overwritten.  G >= 2 per axis. */
int flpr_deposit(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G, int C,
                 const double* const* h_cols, double* d_Q, double* d_B, double* d_sq,
                 void* stream);
/* (5b) The same deposits (and d_sq) from the records of the last
 * flpr_spread / flpr_spread_dkmap call (either precision) with the same d,
 * n, L, msp, nchan and workspace d_spread_ws: one CTA per spreading work
 * item accumulates its points' deposits in shared memory, exact 64-bit
 * fixed point (quantum 2^-62 of each channel's absolute sum), so the
 * result is independent of the order of the points (bitwise reproducible)
 * and no point takes a global atomic of its own.  The deposited channels
 * are the spread's value channels (nchan - ones_channel <= 32; h_cols: their
 * device columns, for the sums of squares in d_sq, taken in point order).  h_ax,
 * h_G: the raw grid as for flpr_deposit; h_m0: per axis the spreading cell
 * of raw-grid node 0 (a placement hint: any value gives the same sums).
 * d = 1 or 2.  d_ws: flpr_deposit_sorted_ws bytes.  No reference
 * counterpart beyond flpr_deposit's. */
size_t flpr_deposit_sorted_ws(int d, int64_t n, const int* h_L, int msp, int nchan);
int flpr_deposit_sorted(int d, int64_t n, const double* d_x, const int* h_L, int msp, int nchan,
                        int ones_channel, const double* const* h_cols,
                        const void* d_spread_ws, size_t spread_ws_bytes,
                        const double* h_ax, const int* h_G, const int* h_m0, double* d_Q,
                        double* d_B, double* d_sq, void* d_ws, size_t ws_bytes, void* stream);
/* quad[h][c] = sum_b sum_pairs B[b][p] m(b+c_k) m(b+c_k') for m (H, M, ny),
 * ny <= 4; d_quad (H, ny) overwritten. */
int flpr_stencil_quad(int d, const int* h_G, int H, int ny, const double* d_m, const double* d_B,
                      double* d_quad, void* stream);
/* The same sums reduced in a fixed order (block partials in d_ws, then one
 * ordered pass): bitwise reproducible. */
size_t flpr_stencil_quad_fixed_ws(int d, const int* h_G, int H, int ny);
int flpr_stencil_quad_fixed(int d, const int* h_G, int H, int ny, const double* d_m,
                            const double* d_B, double* d_quad, void* d_ws, size_t ws_bytes,
                            void* stream);

/* (8) Evaluate one grid (values (M) float64 at every grid point, times
 * nval interleaved value sets, layout (nval, M)) at n points: d_out (nval, n).
 * Clamped multilinear interpolation (interp_optimized.py:60-130); this is
 * the fpp_yhat / fpp interpolant and the final yhat of api.py:760-763. */
int flpr_interp_eval(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G,
                     int nval, const double* d_vals, double* d_out, void* stream);
/* The same evaluation continuing the edge cells' linear functions beyond
 * the grid (cell index clamped, fraction not): scipy's
 * RegularGridInterpolator(method='linear', fill_value=None), which the
 * reference's batch helpers use (batch.py:595-760). */
int flpr_interp_eval_extrap(int d, int64_t n, const double* d_x, const double* h_ax,
                            const int* h_G, int nval, const double* d_vals, double* d_out,
                            void* stream);

/* (8b) Not-a-knot cubic spline interpolation: the 'cubic' GCV / DoF
 * interpolation of api.py:594-600 / api.py:651-657 (regression.py:1015-1020;
 * scipy RegularGridInterpolator(method='cubic', fill_value=None), i.e.
 * make_ndbspl with knots [x0]*4 + x[2:-2] + [x_end]*4 per axis).
 *
 * flpr_spline_prefilter turns grid values into spline coefficients in
 * place.  d_vals: (outer, G_0..G_{d-1}, inner) float64.  d_lu: for each axis
 * in turn, G_a rows of 7 doubles (l3 l2 l1 1/u0 u1 u2 u3): the banded LU
 * factors (no pivoting) of that axis' collocation matrix, zero where a band
 * entry falls outside the matrix.  G >= 4 per axis.
 *
 * flpr_spline_reduce: flpr_interp_reduce with the spline of coefficients
 * d_coef (H, M, ny + R) in place of the multilinear stencil.  d_axes: the
 * raw grid axes concatenated (sum G doubles, strictly increasing, device).
 * Points outside the grid use the end polynomial pieces (fill_value=None).
 *
 * flpr_spline_eval: d_out (nval, n) = spline of d_coef (nval, M) at the
 * points; the cubic final interpolant (interp_method='cubic',
 * api.py:488-503, output_interp_method, api.py:1145-1147). */
int flpr_spline_prefilter(int d, const int* h_G, int64_t outer, int inner, const double* d_lu,
                          double* d_vals, void* stream);
int flpr_spline_reduce(int d, int64_t n, const double* d_x, const double* d_axes, const int* h_G,
                       int H, int ny, int R, const double* d_coef,
                       const double* const* h_ycols, const double* const* h_pcols,
                       double* d_rss, double* d_pdot, double* d_pp, void* stream);
int flpr_spline_eval(int d, int64_t n, const double* d_x, const double* d_axes, const int* h_G,
                     int nval, const double* d_coef, double* d_out, void* stream);

/* (8c) GCV, DoF and the 1-SE choice on the device (regression.py:280-471,
 * regression.py:1276-1354, api.py:73-164), so that the output stage can be
 * enqueued or captured without a host round trip.  d_packed: the reductions
 * of one fit, dual form {sq (C), dots (C, H), quad (H, ny)} (dual = 1) or
 * pointwise form {rss (H, ny), pdot (max(R,1), H), pp (max(R,1))}, C = ny + R;
 * complex responses: ny = 2 dy (real/imaginary interleaved); agg 0/1/2 =
 * gcv_selection 'first'/'average'/'sum'; d_hsum (H): sum over axes of each
 * bandwidth.  d_out (4H) = {gcv_m, gcv_sd, dof, dof_stderr}; d_sel: the
 * 1-SE index, or -1 when no score is finite.  One block.
 * flpr_select_grid: d_gv (ny, M) = d_m[sel][:, :ny] transposed (d_m:
 * (H, M, mstride) float64) and d_s0 (M) = S[0][sel] (S: (ns, H, M), float
 * when s_prec is FLPR_PREC_F32 else double); NaN when sel is out of range. */
int flpr_gcv_select(int H, int ny, int R, int dual, int y_complex, int agg, double n, double dstd,
                    const double* d_packed, const double* d_hsum, double* d_out, int* d_sel,
                    void* stream);
int flpr_select_grid(int64_t M, int ny, int mstride, int H, const double* d_m, const void* d_S,
                     int s_prec, const int* d_sel, double* d_gv, double* d_s0, void* stream);

/* ---------------------------------------------------------------------
 * (9) KDE normalisation and LCV.  Replaces api.py:1059-1133.
 * d_s: (H, M) density sums (float64, epsilon already added).  For each
 * bandwidth: f = max(s / (sum(s) * dxprod), 0) (no division if the sum is
 * not positive), written to d_f (H, M) float64; then f is interpolated at
 * the raw points and the LCV terms log(max(n/(n-1) (f - K0_h/n), 1e-10))
 * are reduced: d_lcv (H, 2) = {sum of the logs, sum of their squared
 * deviations from their mean} (shifted sums, so a constant set of logs
 * gives exactly zero).  h_k0: (H) K0_h values.  The workspace
 * (flpr_kde_ws) also holds a bandwidth-fastest (M, H) copy of the densities
 * that the point-wise interpolation reads.
 * --------------------------------------------------------------------- */
size_t flpr_kde_ws(int64_t n, int H, int64_t M);
int flpr_kde_lcv(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G,
                 int H, const double* d_s, double dxprod, const double* h_k0,
                 double* d_f, double* d_lcv, void* d_ws, size_t ws_bytes, void* stream);

/* (10) Small elementwise helpers used by the variance mode of
 * api.py:390-396 and api.py:771-786. */
int flpr_log_shift(int64_t n, const double* d_in, double shift, double* d_out, void* stream);
/* d_acc[0] = sum_i yraw_i * exp(-yhat_i) */
int flpr_exp_weighted_sum(int64_t n, const double* d_yraw, const double* d_yhat,
                          double* d_acc, void* stream);

/* ---------------------------------------------------------------------
 * (11) Learned bandwidth proposal.  No counterpart in the reference: the
 * reference always sweeps every bandwidth.  A small MLP reads binned moment
 * summaries of a data set and proposes where the GCV minimum lies; a short
 * sweep around the proposal is accepted only when its minimum is interior,
 * otherwise the full sweep runs.
 *
 * flpr_bin_moments: d in {1, 2}; d_stats from flpr_point_stats (min, max
 * per axis).  d_out (3, 4096) float64 receives, per cell of a grid over
 * [min, max] (4096 bins in 1-D, 64 x 64 row-major in 2-D), the count,
 * sum y and sum y^2 (zeroed by the call).
 * --------------------------------------------------------------------- */
int flpr_bin_moments(int d, int64_t n, const double* d_x, const double* d_y,
                     const double* d_stats, double* d_out, void* stream);

/* Feature vectors of B data sets from their binned sums, on the device (the
 * summary learned.summarize forms on the host: per-axis 64-bin count / mean /
 * mean-square profiles of the standardised response, 12 lag-roughness values
 * raw and noise-corrected, the pooled within-cell variance and its log,
 * log10 n, order and dimension one-hots).  d_bins: (B, 3, 4096) from
 * flpr_bin_moments; d_meta: (B, 3) int {d, order, n}; d_fmean / d_fstd: the
 * network's feature standardisation (416 each).  d_feat (optional, may be
 * NULL): (B, 416) FP32 raw features; d_x16: (B, 416) BF16 standardised
 * network inputs.  One CTA per data set. */
int flpr_learned_features(int B, const double* d_bins, const int* d_meta, const float* d_fmean,
                          const float* d_fstd, float* d_feat, void* d_x16, void* stream);

/* Window start of the short local sweep for each of B data sets from the
 * network output d_raw (B): t = clip(raw * t_scale + t_center, 0, ngrid-1)
 * on the canonical grid d_loggrid (ngrid log bandwidths), the target log h
 * linearly interpolated there, the nearest entry c of the data set's own
 * list d_logh (B x lmax, d_nlist[b] valid entries, first on ties) and
 * d_lo[b] = clip(c - refine/2, 0, nlist - refine).  d_t (optional): the
 * unclipped t. */
int flpr_learned_window(int B, const float* d_raw, double t_scale, double t_center, int ngrid,
                        const double* d_loggrid, int lmax, const int* d_nlist,
                        const double* d_logh, int refine, int* d_lo, double* d_t,
                        void* stream);

/* Copy `rows` rows of row_bytes (a multiple of 8) starting at row *d_start
 * (read on the device) of d_src to d_dst: the window's slice of a per-
 * bandwidth table chosen on the device, inside a captured graph. */
int flpr_copy_rows(const void* d_src, void* d_dst, int64_t row_bytes, int rows,
                   const int* d_start, void* stream);

/* Dense ReLU network h_{l+1} = relu(h_l W_l^T + b_l) (no ReLU on the last
 * layer) with dims[0..nlayers].  Parameters are packed per layer as
 * W_l (dims[l+1] x dims[l], row-major) then b_l; d_params32 is the FP32
 * master copy, d_params16 the BF16 copy the products read.  Products are
 * BF16 x BF16 with FP32 accumulation on the tensor cores.
 *
 * flpr_mlp_gemm: C = op(A) op(B) (+ bias[n]) (relu) (* (mask > 0)), with
 * A (M x K) stored row-major (a_trans = 0, A[m*lda+k]) or transposed
 * (a_trans = 1, A[k*lda+m]), B (K x N) stored row-major (b_nk = 0,
 * B[k*ldb+n]) or as N x K (b_nk = 1, B[n*ldb+k]); BF16 operands and mask,
 * FP32 and/or BF16 outputs with leading dimension ldc. */
int flpr_mlp_gemm(int M, int N, int K, const void* d_A, int lda, int a_trans,
                  const void* d_B, int ldb, int b_nk, const float* d_bias, int relu,
                  const void* d_mask, int ldm, float* d_C32, void* d_C16, int ldc,
                  void* stream);
int64_t flpr_mlp_param_count(int nlayers, const int* h_dims);
/* Workspace of flpr_mlp_fwd/flpr_mlp_bwd for `batch` rows: the hidden
 * activations kept for the backward pass and two gradient buffers. */
size_t flpr_mlp_ws(int nlayers, const int* h_dims, int batch);
/* d_x16: (batch, dims[0]) BF16 inputs; d_out: (batch, dims[nlayers]) FP32. */
int flpr_mlp_fwd(int nlayers, const int* h_dims, const void* d_params16,
                 const float* d_params32, int batch, const void* d_x16, float* d_out,
                 void* d_ws, size_t ws_bytes, void* stream);
/* Gradients of sum(d_dout * out) with respect to every parameter, written
 * to d_grad32 (same packing as the parameters).  Uses the activations the
 * preceding flpr_mlp_fwd left in the same workspace. */
int flpr_mlp_bwd(int nlayers, const int* h_dims, const void* d_params16, int batch,
                 const void* d_x16, const float* d_dout, float* d_grad32, void* d_ws,
                 size_t ws_bytes, void* stream);
/* Adam on the FP32 master parameters (an L2 term weight_decay * p is added
 * to the gradient); refreshes the BF16 copy. */
int flpr_mlp_step(int64_t nparams, float* d_params32, void* d_params16, const float* d_grad32,
                  float* d_m, float* d_v, float lr, float beta1, float beta2, float eps,
                  float weight_decay, int step, void* stream);
/* d_loss[0] = mean (y - t)^2; d_dy = 2 (y - t) / batch. */
int flpr_mlp_mse(int batch, const float* d_y, const float* d_t, float* d_dy, float* d_loss,
                 void* stream);
int flpr_to_bf16(int64_t n, const float* d_x, void* d_y, void* stream);

/* Inference of the same network in one launch on the fifth-generation
 * tensor cores (tcgen05.mma, accumulators in tensor memory): each CTA takes
 * 128 rows of the batch through every layer, the activations staying on
 * chip.  Supported shapes (flpr_mlp_infer_supported): input width <= 448
 * and a multiple of 8, every hidden width 256, one output.  d_x16:
 * (batch, dims[0]) BF16; d_out: (batch) FP32.  d_status (optional): set to
 * FLPR_ERR_TIMEOUT if a bounded wait of the kernel ran out (the outputs are
 * then not written).  No reference counterpart (the learned proposal is not
 * part of the reference). */
int flpr_mlp_infer_supported(int nlayers, const int* h_dims);
int flpr_mlp_infer(int nlayers, const int* h_dims, const void* d_params16,
                   const float* d_params32, int batch, const void* d_x16, float* d_out,
                   int* d_status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FASTLPR_B200_H */
