/*
 * algotom_b200 -- C ABI of the B200 filtered-back-projection library.
 *
 * These are the entry points a foreign-function binding of algotom's FBP /
 * BPF hot path (algotom 1.6.0, algotom/rec/reconstruction.py) calls.  They
 * take plain device pointers, element strides and sizes; the caller owns
 * every buffer and the library never frees caller memory.  Every call is
 * asynchronous on the given stream (cudaStream_t passed as void*, NULL for
 * the legacy default stream) and re-entrant per stream.
 *
 * Return value: 0 on success, a negative ATB_E* code otherwise; the message
 * of the calling thread's last failure is atb_last_error().  The library
 * never aborts and never traps the device.
 *
 * Layouts follow the reference: a sinogram stack is [nrow angles][nslice]
 * [ncol detector pixels] and a reconstruction stack is [ncol rows (y)]
 * [nslice][ncol columns (x)].  Row and slice strides are in elements; the
 * detector (x) axis is contiguous.
 */
#ifndef ALGOTOM_B200_H
#define ALGOTOM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define ATB_OK 0
#define ATB_EINVAL (-1)   /* bad argument: size, stride, pointer, enum */
#define ATB_ECUDA (-2)    /* a CUDA runtime call failed */
#define ATB_ERANGE (-3)   /* size beyond what this build supports */

/* element types of sinogram storage */
#define ATB_F32 0
#define ATB_F16 1
#define ATB_BF16 2
#define ATB_U16 3  /* raw detector counts (atb_flat_log input only) */

/* numpy.pad modes along the detector axis (reconstruction.py:146) */
#define ATB_PAD_EDGE 0
#define ATB_PAD_CONSTANT 1     /* constant_values = 0 */
#define ATB_PAD_REFLECT 2
#define ATB_PAD_SYMMETRIC 3
#define ATB_PAD_WRAP 4
#define ATB_PAD_LINEAR_RAMP 5  /* end_values = 0 */
#define ATB_PAD_MEAN 6
#define ATB_PAD_MAXIMUM 7
#define ATB_PAD_MINIMUM 8
#define ATB_PAD_MEDIAN 9

/* slice metrics of the centre search */
#define ATB_METRIC_ENTROPY 0
#define ATB_METRIC_SHARPNESS 1

/* Library version as major*10000 + minor*100 + patch. */
int atb_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char *atb_last_error(void);

/*
 * Asynchronous strided copy of `height` rows of `width` bytes (pitches in
 * bytes), kind 0 host->device, 1 device->host, 2 device->device; one
 * cudaMemcpy2DAsync.  Used to stream slabs of slices of a host stack
 * [nrow][nslice][ncol] through the device while the previous slab computes
 * (the reference copies whole chunks synchronously at each kernel launch,
 * reconstruction.py:476-481).
 */
int atb_copy_2d(void *dst, int64_t dst_pitch, const void *src,
                int64_t src_pitch, int64_t width, int64_t height, int kind,
                void *stream);

/*
 * Transform length n the row filter uses for a detector width `ncol` and
 * pad `pad`, the cheaper (by a flop count of its FFT stages) of
 * N = ncol + 2 pad itself, when N has no prime factor above 13 (the
 * reference's own transform: 2860 = 4 5 11 13 at 2560 pixels, pad 150), and
 * the 7-smooth lengths n >= N + ncol - 1 (a circular convolution of length
 * n then reproduces the one of length N exactly on the cropped window).
 * At most 16384; a negative code if no length fits.
 */
int atb_filter_length(int ncol, int pad);

/*
 * The twiddle table of the row filter's transforms of length n (a length
 * atb_filter_length returns), written to HOST memory: n complex64 values,
 * the twiddles of each FFT stage in the order the kernel reads them
 * (exp(-2 pi i r k / (Ns R)) for stage radix R after sub-transforms of
 * length Ns), computed in FP64.  The caller copies it to the device once
 * per length and passes it as `twiddle`.
 */
int atb_filter_twiddles(int n, void *host_out);

/*
 * Padded ramp-and-window filter of every row of a sinogram stack, with the
 * optional -log folded in; replaces apply_ramp_filter
 * (algotom/rec/reconstruction.py:118-153) and the -log pre-step
 * (reconstruction.py:431-436; values <= 0 read as 1, i.e. give 0).
 *
 *   src      float32 [nrow][nslice][ncol] at src_row_stride / src_slice_stride
 *   pad      detector padding on each side; pad_mode one of ATB_PAD_*
 *   spec     complex64 [spec_rows][fft_len]: spectrum of the periodised
 *            real kernel, already scaled by 1 / fft_len.  spec_rows = 1 (one
 *            kernel for every row) or nrow (one kernel per angle; then two
 *            slices of one angle share a transform)
 *   twiddle  complex64 [fft_len]: atb_filter_twiddles(fft_len) on the device
 *   fft_len  a length with fft_len == ncol + 2 pad (no prime factor above
 *            13) or fft_len >= 2 ncol + 2 pad - 1 (7-smooth), at most 16384;
 *            atb_filter_length gives the cheapest
 *   dst      [nrow][nslice][ncol] of dst_dtype (ATB_F32/F16/BF16) at
 *            dst_row_stride / dst_slice_stride
 */
int atb_filter_rows(const float *src, int64_t src_row_stride,
                    int64_t src_slice_stride, int nrow, int nslice, int ncol,
                    int pad, int pad_mode, int apply_log, const void *spec,
                    int spec_rows, const void *twiddle, int fft_len, void *dst,
                    int dst_dtype, int64_t dst_row_stride,
                    int64_t dst_slice_stride, void *stream);

/*
 * One single-slice sinogram of a batched filter launch (device pointers
 * inside).  pair_offset: index of its first row pair in the launch (the
 * running sum of (nrow + 1) / 2 over the items before it).
 */
typedef struct {
  const float *src;         /* [nrow][ncol] */
  int64_t src_row_stride;
  void *dst;                /* [nrow][ncol] of the launch's dst_dtype */
  int64_t dst_row_stride;
  const void *spec;         /* as atb_filter_rows, spec_rows = 1 */
  int nrow;
  int ncol;
  int pad;
  int pair_offset;
} atb_filter_item;

/*
 * atb_filter_rows over a batch of single-slice sinograms of uneven width
 * and angle count that share the transform length fft_len, in ONE launch: CTA p
 * filters row pair p - pair_offset of the item whose pair range holds p.
 * The uneven-batch counterpart of the reference's per-slice filtering
 * (reconstruction.py:460-475); no counterpart of the batching itself.
 *
 *   items     DEVICE array [nitems], ordered by pair_offset (0 first)
 *   npairs    total row pairs (sum of (nrow + 1) / 2)
 *   pad_mode, apply_log, twiddle, fft_len, dst_dtype as atb_filter_rows;
 *             every item needs fft_len == ncol + 2 pad or fft_len >=
 *             2 ncol + 2 pad - 1, its spectrum built for fft_len (items
 *             longer than fft_len are skipped)
 */
int atb_filter_rows_batch(const atb_filter_item *items, int nitems,
                          int npairs, int pad_mode, int apply_log,
                          const void *twiddle, int fft_len, int dst_dtype,
                          void *stream);

/*
 * Elementwise -log of a float32 sinogram stack, values <= 0 read as 1;
 * the BPF pre-step (reconstruction.py:632-637).  dst may equal src.
 */
int atb_neg_log(const float *src, int64_t src_row_stride,
                int64_t src_slice_stride, int nrow, int nslice, int ncol,
                float *dst, int64_t dst_row_stride, int64_t dst_slice_stride,
                void *stream);

/*
 * Linear-interpolation back-projection of a stack of sinograms that share
 * angles and centre; replaces __back_projection_gpu_kernel /
 * back_projection_gpu (reconstruction.py:156-226),
 * __back_projection_gpu_chunk_kernel / back_projection_gpu_chunk
 * (reconstruction.py:229-304) and back_projection_cpu
 * (reconstruction.py:307-359), fused with the circle mask and the
 * pi/(nrow-1) scale of fbp_reconstruction (reconstruction.py:488-493).
 *
 *   sino     [nrow][nslice][ncol] of sino_dtype at the given strides
 *   trig     float64 [nrow][2] = (cos(-a), sin(-a)) for the float32-rounded
 *            angles a
 *   center   float32-rounded rotation centre, as a double
 *   edge_pad 0: positions outside [0, ncol-1] add nothing (FBP);
 *            1: they add the nearest edge sample (BPF)
 *   mask_r2  < 0: no mask; else pixels with (x-c)^2 + (y-c)^2 > mask_r2,
 *            c = ncol/2 (integer division), are written as 0
 *   scale    multiplies every written pixel
 *   out      float32 [ncol][nslice][ncol] at out_row_stride / out_slice_stride
 *   flags    bit 0: per-angle compensated (Kahan) accumulation instead of
 *            the default chunked Kahan (FP32 partials over a chunk of angles,
 *            compensated across chunks);
 *            bit 1: back-project the derivative of the interpolant with
 *            respect to p instead of its value: s[d+1] - s[d] at
 *            d = floor(p), plus the two detector-edge steps (+s[0] at
 *            p = 0, -s[ncol-1] at p = ncol-1) smoothed over one bin; this
 *            is the derivative of the back-projection with respect to the
 *            centre (no counterpart in the reference; used by the autograd
 *            path; edge_pad must be 0);
 *            bits 2-3: tile variant for single-slice launches: 0 = 64 x 64
 *            pixels on 256 threads, 1 = 32 x 32 on 128 threads (chosen by the
 *            autotuner; stacks of 2 or more slices always use 64 x 32 tiles);
 *            bit 4: stage the detector windows with cp.async even where
 *            TMA box loads are used by default (CTAs of 2 or 4 slices with a
 *            16-byte aligned base, strides and row length); same results;
 *            bit 5 (tests of the bounded waits only): the first CTA of a
 *            TMA-staged launch arms its first window wait for 16 bytes more
 *            than its copies deliver, and every wait gives up after 4096
 *            polls instead of about 2^20.  That wait then runs out with every
 *            copy complete: the CTA sets bit 0 of atb_backproject_status
 *            and leaves its tile unwritten; the other tiles are unaffected
 */
int atb_backproject(const void *sino, int sino_dtype, int64_t sino_row_stride,
                    int64_t sino_slice_stride, int nrow, int nslice, int ncol,
                    const double *trig, double center, int edge_pad,
                    double mask_r2, float scale, float *out,
                    int64_t out_row_stride, int64_t out_slice_stride,
                    int flags, void *stream);

/*
 * Back-projection of ONE sinogram at ncenter rotation centres
 * center + m * spacing (m = 0 .. ncenter-1, spacing a whole number of
 * pixels); replaces the per-candidate reconstructions of a centre search
 * (_find_center_based_slice_metric, reconstruction.py:1254-1346, through
 * _reconstruct_slice, :1177-1208) for candidates whose float32 centres
 * differ by whole pixels.  Image m equals atb_backproject of the sinogram
 * at centre center + m * spacing (same positions, pairs and edge decisions;
 * only the grouping of the FP32 partial sums differs).  Centres at a
 * non-integer step, e.g. 0.25, form one such progression per residue:
 * call once per residue with out offset by the residue's image.
 *
 *   sino      float32 [nrow][ncol] at sino_row_stride
 *   trig, edge_pad, scale, flags (bit 4)   as atb_backproject
 *   center    the float32-rounded first centre, as a double; every centre
 *             center + m * spacing must lie in [0, ncol)
 *   spacing   1 .. 56
 *   mask_r2   as atb_backproject, the same for every centre
 *   out       float32 image m at out + m * out_center_stride, rows
 *             out_row_stride apart
 */
int atb_backproject_centers(const float *sino, int64_t sino_row_stride,
                            int nrow, int ncol, const double *trig,
                            double center, int spacing, int ncenter,
                            int edge_pad, double mask_r2, float scale,
                            float *out, int64_t out_row_stride,
                            int64_t out_center_stride, int flags,
                            void *stream);

/*
 * Status word of the back-projection kernels: bit 0 is set when a CTA gave
 * up waiting (after about 70 ms) for a TMA window load and left its tile
 * unwritten.  Returns the word (0 = no such event since the last reset) and
 * clears it when reset != 0; negative on a CUDA error.  Synchronises with
 * the device.
 */
int atb_backproject_status(int reset);

/*
 * Forward (Radon) projection that is the exact adjoint of atb_backproject
 * without edge padding: out[i][k][d] = sum over pixels of
 * img[y][k][x] * hat(p_i(y, x) - d) over positions inside [0, ncol-1].
 * The transpose of the reference back-projector
 * (algotom/rec/reconstruction.py:156-190, 307-359), which has no adjoint of
 * its own; it gives the gradient of a back-projection with respect to its
 * sinogram, and is the projector of model-based reconstruction.
 *
 *   img   float32 [ncol][nslice][ncol] at img_row_stride / img_slice_stride
 *   trig, center as for atb_backproject
 *   out   float32 [nrow][nslice][ncol] at out_row_stride / out_slice_stride
 *   workspace  device scratch of at least atb_radon_workspace(nslice, ncol)
 *         bytes (a transposed copy of the image, read for angles whose rays
 *         cross the image columns more steeply than its rows)
 *
 * Deterministic: the same inputs give the same bits.
 */
int64_t atb_radon_workspace(int nslice, int ncol);
int atb_radon_adjoint(const float *img, int64_t img_row_stride,
                      int64_t img_slice_stride, int nrow, int nslice,
                      int ncol, const double *trig, double center, float *out,
                      int64_t out_row_stride, int64_t out_slice_stride,
                      void *workspace, int64_t workspace_bytes, void *stream);

/*
 * One single-slice back-projection of a batch (device pointers inside).
 * Field meanings as in atb_backproject; the sinogram is float32.
 */
typedef struct {
  const float *sino;        /* [nrow][ncol] */
  int64_t sino_row_stride;
  const double *trig;       /* [nrow][2] */
  float *out;               /* [ncol][ncol] */
  int64_t out_row_stride;
  double center;
  double mask_r2;
  float scale;
  int nrow;
  int ncol;
  int edge_pad;
} atb_bp_item;

/*
 * Host-side work list of a batch for atb_backproject_batch: one entry per
 * (item, pixel tile), item index << 16 | tile, items ordered by angle
 * count, largest first (longest-processing-time order).  Tiles are
 * 64 x 64 pixels for variant 0 and 32 x 32 for variant 1 (as the flags of
 * atb_backproject); at most 65536 tiles per item (ncol <= 16384 or 8192)
 * and 65536 items.  With units == NULL returns the number of entries;
 * otherwise fills up to `capacity` and returns the count.  No counterpart in
 * the reference, which loops over slices on the host
 * (reconstruction.py:482-487).
 */
int atb_bp_batch_plan(const atb_bp_item *items, int nitems, int *units,
                      int capacity, int variant);

/*
 * Back-projection of a batch of single-slice sinograms of uneven width,
 * angle count and centre in one persistent launch: each CTA pulls work
 * units from `counter` until `units` is exhausted.  Batched counterpart of
 * __back_projection_gpu_kernel (reconstruction.py:156-190), one launch for
 * what the reference does with one launch per call.
 *
 *   items    device array [nitems] of atb_bp_item
 *   units    device array [nunits] from atb_bp_batch_plan
 *   counter  device scratch, two int32, zero before the first call; the
 *            kernel returns it to zero, so a CUDA graph can replay the launch
 *   max_ctas 0: as many CTAs as fit (2 per SM for variant 0, 4 for
 *            variant 1); otherwise at most this many CTAs
 *   variant  tile variant the units were planned for (0 or 1)
 *
 * Calls that share `counter` must not overlap on the device.
 */
int atb_backproject_batch(const atb_bp_item *items, int nitems,
                          const int *units, int nunits, int *counter,
                          int max_ctas, int variant, void *stream);

/*
 * atb_backproject_batch for callers that cannot allocate device memory.
 * No counterpart in the reference (it is an addition of this library).
 *
 * For a caller that owns device buffers for its sinograms, angle tables and
 * outputs but may not call cudaMalloc -- a plugin whose host application
 * accounts for every device byte, a loop that cannot afford cudaMalloc's
 * implicit synchronisation, a foreign-language caller with no CUDA runtime
 * of its own.  Takes the item table in HOST memory (device pointers inside)
 * and keeps the work list, item table and counter in a fixed __device__
 * array of this library (about 4.4 MB, held by every GPU that loads the
 * library until the process exits).  It allocates nothing.  The table is
 * read during the call only: its entries travel to the device inside the
 * parameters of the launches the call enqueues, and the work list is built
 * on the device, so the caller may reuse or free the host table as soon as
 * the call returns, and the call does not wait for earlier work on the
 * stream.  Items are accepted as atb_backproject_batch accepts them (any
 * centre).
 *
 *   items     host array [nitems], nitems <= 4096; ncol <= 16384 per item
 *   max_ctas  as atb_backproject_batch
 *
 * Limits: at most 4096 items and 1048576 tiles of 64 x 64 pixels in total;
 * larger batches are rejected with ATB_ERANGE before any device work.
 * The first call on a device looks up the array's device address (once per
 * device, with that device current).  Every call reuses the same array and overwrites the previous
 * call's table: calls that overlap on the device (on different streams, or
 * from different host threads without ordering) race on it.
 */
int atb_backproject_batch_noalloc(const atb_bp_item *items, int nitems,
                                  int max_ctas, void *stream);

/*
 * Transform length T the 2-D BPF filter uses for a slice of ncol x ncol
 * padded by pad on every side: N = ncol + 2 pad when all prime factors of
 * N are at most 13, else the smallest M >= N + ncol - 1 whose prime
 * factors are at most 7 (a circular convolution of that length reproduces
 * the N-periodic one exactly on the cropped slice).  ATB_ERANGE above 7168.
 */
int atb_bpf_filter2d_length(int ncol, int pad);

/* Device workspace bytes of atb_bpf_filter2d processing `pairs` slice
 * pairs at once (it processes the stack in groups of as many pairs as the
 * workspace it is given holds; one pair is the minimum). */
int64_t atb_bpf_filter2d_workspace(int ncol, int pad, int pairs);

/*
 * 2-D circular ramp filter of every slice of a back-projection stack, with
 * the circle mask and scale of BPF fused; replaces
 * apply_circular_ramp_filter (algotom/rec/reconstruction.py:527-560) as
 * bpf_reconstruction applies it per slice, then its mask and
 * pi/(nrow-1) scale (reconstruction.py:675-684).  Each slice is padded to
 * N x N with numpy's mode (both axes, axis 0 first as numpy does), filtered
 * with the spectrum, cropped; FP64 transforms of this library, two slices
 * per complex transform.
 *
 *   src       float32 [ncol (y)][nslice][ncol (x)] at the given strides
 *             (the layout atb_backproject writes)
 *   pad, pad_mode  as apply_circular_ramp_filter (ATB_PAD_*)
 *   spectrum  device [T][T] with T = atb_bpf_filter2d_length(ncol, pad),
 *             stored transposed ([kx][ky]) and scaled by 1 / T^2: for
 *             T = N the Hermitian part (H(k) + conj(H(-k))) / 2 of
 *             H = ifftshift(W2); for T > N the 2-D transform of the
 *             N-periodic kernel ifft2 of that part, placed on the T x T
 *             torus at the lags [pad - N + 1, pad + ncol - 1] of each axis.
 *             float64 when spectrum_complex == 0, else complex128
 *   twiddle   complex128 [T]: exp(-2 pi i m / T)
 *   mask_r2   < 0: no mask; else pixels with (x-c)^2 + (y-c)^2 > mask_r2,
 *             c = ncol/2, are written as 0
 *   scale     multiplies every written pixel
 *   dst       float32 [ncol][nslice][ncol] at the given strides; may be src
 *   workspace device scratch of at least
 *             atb_bpf_filter2d_workspace(ncol, pad, 1) bytes
 */
int atb_bpf_filter2d(const float *src, int64_t src_row_stride,
                     int64_t src_slice_stride, int nslice, int ncol, int pad,
                     int pad_mode, const void *spectrum, int spectrum_complex,
                     const void *twiddle, double mask_r2, float scale,
                     float *dst, int64_t dst_row_stride,
                     int64_t dst_slice_stride, void *workspace,
                     int64_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------- */
/* Centre search by slice metrics (find_center_based_slice_metric,        */
/* algotom/rec/reconstruction.py:1212-1458).  The candidate centres are   */
/* reconstructed by one atb_backproject_batch launch whose items share    */
/* the filtered sinogram; these entry points cover the steps around it.   */
/* ---------------------------------------------------------------------- */

/*
 * scipy.ndimage.gaussian_filter1d(x, sigma, axis=1) of float32 rows, mode
 * "reflect"; replaces the smoothing of the sinogram before a search
 * (reconstruction.py:1317-1318).  Same float32 results as scipy.
 *
 *   weights   device float64 [radius + 1]: the half kernel w[0..radius] of
 *             the unit-sum sampled Gaussian, radius = int(4 sigma + 0.5)
 *   dst       must not overlap src; radius <= 8192, ncol <= 65535 * 256
 *   to_int    nonzero: each output is truncated toward zero, the value scipy
 *             stores when the input array has an integer dtype (the counts
 *             are passed as exact float32 integers)
 */
int atb_gaussian_rows(const float *src, int64_t src_row_stride, int nrow,
                      int ncol, const double *weights, int radius,
                      float *dst, int64_t dst_row_stride, int to_int,
                      void *stream);

/*
 * The same filter down the columns of nimg float32 images
 * (gaussian_filter1d along axis 1 of a [nimg, nrow, ncol] stack), the first
 * pass of the projection smoothing gaussian_filter(projections,
 * (0, sigma, sigma)) before a vertical-slice centre search
 * (vertrec.py:1348-1349; the second pass is atb_gaussian_rows).  Same
 * float32 results as scipy.
 *
 *   weights   as atb_gaussian_rows; radius <= 700 (the strip with its halo
 *             fits in shared memory)
 *   dst       must not overlap src; nrow * row_stride < 2^31
 *   to_int    as atb_gaussian_rows
 */
int atb_gaussian_cols(const float *src, int64_t src_img_stride,
                      int64_t src_row_stride, int nimg, int nrow, int ncol,
                      const double *weights, int radius, float *dst,
                      int64_t dst_img_stride, int64_t dst_row_stride,
                      int to_int, void *stream);

/*
 * scipy.ndimage.zoom(x, zoom, order=1, mode="nearest") of a float32 image
 * to out_rows x out_cols (the caller computes round(n * zoom)); replaces
 * the coarse-search resize (reconstruction.py:1426-1428).  Same float32
 * results as scipy.  out_rows <= 65535.
 */
int atb_zoom_linear(const float *src, int64_t src_row_stride, int in_rows,
                    int in_cols, float *dst, int64_t dst_row_stride,
                    int out_rows, int out_cols, void *stream);

/*
 * out2 = (min, max) of a float32 image (both NaN if any pixel is NaN), the
 * entropy normalisation range (reconstruction.py:1327-1330).
 *
 *   work   device scratch of 12 bytes
 *   out2   device float32 [2]
 */
int atb_image_range(const float *img, int64_t row_stride, int rows, int cols,
                    void *work, float *out2, void *stream);

/* Bytes of device scratch atb_slice_metric needs (0 for a bad argument). */
int64_t atb_slice_metric_workspace(int nimg, int rows, int cols, int metric);

/*
 * One metric per image of a batch: ATB_METRIC_ENTROPY, the histogram
 * entropy of the image normalised by (nmin, nmax) to uint8 levels
 * (reconstruction.py:1212-1221 with the normalisation of :1243-1245), or
 * ATB_METRIC_SHARPNESS, the mean gradient magnitude (:1224-1229; needs
 * rows, cols >= 2).  Deterministic.
 *
 *   imgs      float32 [nimg] images of rows x cols at img_stride, row_stride
 *   work      device scratch of atb_slice_metric_workspace() bytes
 *   out       device float64 [nimg]
 */
int atb_slice_metric(const float *imgs, int64_t img_stride,
                     int64_t row_stride, int nimg, int rows, int cols,
                     int metric, float nmin, float nmax, void *work,
                     int64_t work_bytes, double *out, void *stream);

/*
 * The histogram entropy of float64 images, normalised in FP64: the metric
 * of find_center_vertical_slice (vertrec.py:1389-1392) on slices that the
 * "after" ramp filter leaves in float64.  Arguments as atb_slice_metric
 * (work: atb_slice_metric_workspace(nimg, rows, cols, ATB_METRIC_ENTROPY)
 * bytes).
 */
int atb_slice_entropy64(const double *imgs, int64_t img_stride,
                        int64_t row_stride, int nimg, int rows, int cols,
                        double nmin, double nmax, void *work,
                        int64_t work_bytes, double *out, void *stream);

/* ---------------------------------------------------------------------- */
/* Vertical slices (algotom/rec/vertrec.py)                               */
/* ---------------------------------------------------------------------- */

/*
 * Back-projection of projections onto vertical slices; replaces
 * vertical_back_projection_cpu / vertical_back_projection_gpu
 * (vertrec.py:53-109, 175-252) and their _chunk forms for several slices
 * (vertrec.py:112-172, 255-335).  Slice s is a line of npts points
 * (x, y) in the horizontal plane; for every detector row i and point j
 *
 *   acc[s][i][j] += sum_n value(proj[n][i][.], x cos a_n + y sin a_n + center)
 *
 * with the reference's interpolation, inclusive bounds [0, width-1] and
 * optional edge padding.  Positions in FP64, interpolation FP32, sums over
 * 32 angles FP32, accumulation FP64.  Deterministic.
 *
 *   proj    float32 [nproj][height][width] at proj_stride / row_stride
 *           (height * row_stride < 2^31)
 *   trig    float64 [nproj][2] = (cos a, sin a)  (note: +a, not -a)
 *   points  float64 [nline][npts][2] = (x, y), line_stride between lines
 *           (in points)
 *   line_centers  device float64 [nline]: a centre per line (candidate
 *           centres of one slice, find_center_vertical_slice), or NULL:
 *           every line uses `center`
 *   acc     float64 [nline][height][npts], added to (not overwritten)
 *   work    device scratch of up to atb_vertical_workspace() bytes, or
 *           NULL: with it, the angles are also split over CTAs when the
 *           output alone is too small to fill the GPU (fewer bytes give a
 *           smaller split)
 */
int atb_vertical_backproject(const float *proj, int64_t proj_stride,
                             int64_t row_stride, int nproj, int height,
                             int width, const double *trig,
                             const double *points, int64_t line_stride,
                             int npts, int nline, double center,
                             const double *line_centers, int edge_pad,
                             double *acc, int64_t acc_line_stride,
                             int64_t acc_row_stride, void *work,
                             int64_t work_bytes, void *stream);

/* Bytes of scratch that let atb_vertical_backproject split its angles
 * fully (0: no split is useful, or a bad argument). */
int64_t atb_vertical_workspace(int nproj, int height, int npts, int nline);

/*
 * Flat-field correction and -log of a chunk of projections; replaces the
 * pre-step of vertical_reconstruction* (vertrec.py:594-606):
 *   v = (src - dark) / flat_dark   (when dark / flat_dark are given)
 *   v = -log(v), values <= 0 replaced by 1 first (when apply_log)
 * in float32.  *nonpos (device, not cleared) is increased by the number of
 * replaced values, for the reference's warning.
 *
 *   src        ATB_F32 or ATB_U16 [nproj][height][width]
 *   dark, flat_dark  float32 [height][width] at field_row_stride, both or
 *              neither (flat_dark = flat - dark with zeros set to 1)
 */
int atb_flat_log(const void *src, int src_dtype, int64_t src_proj_stride,
                 int64_t src_row_stride, int nproj, int height, int width,
                 const float *dark, const float *flat_dark,
                 int64_t field_row_stride, int apply_log, float *dst,
                 int64_t dst_proj_stride, int64_t dst_row_stride,
                 unsigned *nonpos, void *stream);

/* ---------------------------------------------------------------------- */
/* 360-degree sinograms (algotom/prep/conversion.py)                      */
/* ---------------------------------------------------------------------- */

/*
 * scipy.ndimage.shift(x, (0, shift), mode="nearest") of float32 rows
 * (cubic spline, the sub-pixel shift of stitch_image and
 * convert_sinogram_180_to_360, conversion.py:104-110, 389-391); with
 * `flip` the rows are mirrored left-right first (np.fliplr).  shift == 0
 * copies.  ncol <= 16384.
 */
int atb_shift_rows(const float *src, int64_t src_row_stride, int nrow,
                   int ncol, double shift, int flip, float *dst,
                   int64_t dst_row_stride, void *stream);

/*
 * The centring of __dfi_handle_sinogram (reconstruction.py:756-770): rows
 * of ncol_src samples padded on the right with their last sample to ncol
 * columns (np.pad(mode="edge"), one column for an even width), then
 * shifted as atb_shift_rows does.  ncol_src <= ncol <= 16384.
 */
int atb_shift_rows_ext(const float *src, int64_t src_row_stride, int nrow,
                       int ncol_src, int ncol, double shift, float *dst,
                       int64_t dst_row_stride, void *stream);

/*
 * The row work of extend_sinogram (conversion.py:425-454): optional -log,
 * the sub-pixel shift (0: none), the linear ramp over `overlap` columns on
 * `side` (1: right, 0: left), edge padding to 2 ncol - overlap columns and
 * the factor 2.  dst rows hold 2 ncol - overlap floats.  ncol <= 16384.
 */
int atb_extend_rows(const float *src, int64_t src_row_stride, int nrow,
                    int ncol, int apply_log, double shift, int overlap,
                    int side, float *dst, int64_t dst_row_stride,
                    void *stream);

/* ---------------------------------------------------------------------- */
/* Direct Fourier inversion (dfi_reconstruction, reconstruction.py:687)   */
/* ---------------------------------------------------------------------- */

/*
 * B-spline coefficients of order 3 or 5 along many strided lines;
 * replaces scipy.ndimage.spline_filter1d inside the map_coordinates of
 * dfi_reconstruction (reconstruction.py:776-781, order 5, "reflect") and
 * the shift along angles of __dfi_handle_angles (:746, order 3, "wrap").
 * Applied as the filter's symmetric impulse response (2 x 48 taps for
 * order 5, 2 x 32 for order 3), exact to below 1e-17 relative.
 *
 *   src, dst  float64, not overlapping; line L = (outer, comp) starts at
 *             + (L / ncomp) * line_stride + (L % ncomp), elements
 *             elem_stride apart (strides in doubles); ncomp = 2 walks the
 *             real and imaginary parts of interleaved complex data.  Either
 *             the elements (elem_stride == ncomp) or the lines
 *             (line_stride == ncomp) must be contiguous.
 *   boundary  0: half-sample symmetric extension (scipy's "reflect"; also
 *             "nearest" after 12 edge samples of padding),
 *             1: whole-sample symmetric (scipy's "mirror" and "wrap")
 */
int atb_spline_prefilter(const double *src, double *dst, int64_t line_stride,
                         int64_t elem_stride, int nlines, int ncomp, int n,
                         int order, int boundary, void *stream);

/*
 * Regrid the polar spectrum of a sinogram onto the width x width Cartesian
 * frequency grid; replaces generate_mapping_coordinate
 * (reconstruction.py:687-728) plus util.mapping(order=5, mode="reflect")
 * and the unit circle mask in __dfi_single_slice (:767-787).
 *
 *   coef   complex128 [nrow][width]: quintic B-spline coefficients of the
 *          centred row spectra (atb_spline_prefilter, order 5, boundary 0,
 *          along both axes)
 *   out    complex128 [width][width] in ifftshift order: frequency grid
 *          point (i, j) at ((i - width/2) mod width, (j - width/2) mod
 *          width), ready for the inverse 2-D transform
 */
int atb_dfi_regrid(const double *coef, int nrow, int width, double *out,
                   void *stream);

/*
 * __dfi_handle_angles (reconstruction.py:731-749), first half: with fold,
 * the 360-degree fold (n = nrow_in / 2 + 1 rows, row r = (row r + row
 * nrow_in - n + r mirrored left-right) / 2 in float32; else n = nrow_in),
 * then the stack the angle shift runs on: rows 0 .. n - 2 followed by all
 * n rows mirrored, 2 n - 1 rows, widened to float64.
 *
 *   src  float32, row r of slice k at src + k src_slice_stride
 *        + r src_row_stride, ncol samples
 *   dst  float64, row i of slice k at dst + k dst_slice_stride
 *        + i dst_row_stride
 */
int atb_dfi_angle_stack(const float *src, int64_t src_row_stride,
                        int64_t src_slice_stride, int nrow_in, int nslice,
                        int ncol, int fold, double *dst,
                        int64_t dst_row_stride, int64_t dst_slice_stride,
                        void *stream);

/*
 * Second half: scipy.ndimage.shift(stack, (shift, 0), order=3,
 * mode="wrap")[:nout] (reconstruction.py:746) from the stack's cubic
 * B-spline coefficients along the rows (atb_spline_prefilter, order 3,
 * boundary 1): coordinate i - shift wrapped into [0, m - 1] with period
 * m - 1, mirrored tap indices, rounded to float32.  flip: reverse rows and
 * columns (the flipud(fliplr(.)) of descending angles, :747-748).
 */
int atb_wrap_shift_rows(const double *coef, int64_t coef_row_stride,
                        int64_t coef_slice_stride, int m, int nslice,
                        int ncol, double shift, int nout, int flip,
                        float *dst, int64_t dst_row_stride,
                        int64_t dst_slice_stride, void *stream);

/*
 * The Fourier transforms of DFI as Bluestein transforms of the padded
 * width w (any w >= 2 with a power-of-two M >= 2 w - 1, M <= 8192; w =
 * 3841 at 2560 detector pixels), FP64, this library's own FFT.
 *
 * atb_dfi_fft_length: M for width w (ATB_ERANGE beyond 8192).
 * atb_dfi_fft_setup: from host-made tables on the device, chirp complex128
 *   [w] = exp(i pi (m^2 mod 2w) / w) and twiddle complex128 [M] =
 *   exp(-2 pi i m / M), fills bfwd and binv (complex128 [M] each): the
 *   chirp kernels' transforms that the other calls read.
 */
int atb_dfi_fft_length(int w);
int atb_dfi_fft_setup(int w, const void *chirp, const void *twiddle,
                      void *bfwd, void *binv, void *stream);

/*
 * Padding, -log and row transform of __dfi_single_slice and
 * dfi_reconstruction (reconstruction.py:767-770, 774-776, 885-890):
 * every row of n float32 samples padded to w = n + 2 pad columns with
 * NumPy's pad_mode (ATB_PAD_*, end and constant values 0, statistics over
 * the whole row), with apply_log -log'ed (values <= 0 give 0; their count
 * over the padded rows is written to *nonpositive when it is not null),
 * then fftshift(fft(ifftshift(row))) * window (window float64 [w] or null)
 * as complex128.  Rows r of slice k: src + k src_slice_stride
 * + r src_row_stride, dst + k dst_slice_stride + r dst_row_stride
 * (strides in floats and in complex values).
 */
int atb_dfi_rows(const float *src, int64_t src_row_stride,
                 int64_t src_slice_stride, int nrow, int nslice, int n,
                 int pad, int pad_mode, int apply_log, const double *window,
                 int *nonpositive, const void *chirp, const void *twiddle,
                 const void *bfwd, const void *binv, void *dst,
                 int64_t dst_row_stride, int64_t dst_slice_stride,
                 void *stream);

/*
 * Regridding, inverse 2-D transform, crop and mask of __dfi_single_slice
 * and dfi_reconstruction (reconstruction.py:776-787, 895-904): from the
 * quintic B-spline coefficients of the polar spectrum (complex128 [nrow]
 * [w] per slice, atb_spline_prefilter along both axes), the Cartesian
 * spectrum is regridded row by row as atb_dfi_regrid does, inverted,
 * cropped to [pad, pad + ncol) on both axes, divided by w^2 and masked by
 * the circle of radius^2 mask_r2 about ncol / 2 (mask_r2 < 0: none);
 * float64 out (float32 with out_f32).  Pixel (a, b) of slice k at out
 * + k out_slice_stride + a out_row_stride + b (in elements).  workspace:
 * atb_dfi_inverse_workspace(w, ncol, nslice) bytes.
 */
int64_t atb_dfi_inverse_workspace(int w, int ncol, int nslice);
int atb_dfi_inverse(const void *coef, int64_t coef_row_stride,
                    int64_t coef_slice_stride, int nrow, int nslice, int w,
                    int pad, int ncol, double mask_r2, const void *chirp,
                    const void *twiddle, const void *bfwd, const void *binv,
                    void *out, int64_t out_row_stride,
                    int64_t out_slice_stride, int out_f32, void *workspace,
                    int64_t workspace_bytes, void *stream);

/*
 * FP64 ramp filter of rows, as a vertical reconstruction applies it after
 * its back-projection (algotom/rec/vertrec.py:677-684 and
 * __apply_ver_ramp_filter, :697-706): every float64 row of ncol samples
 * padded with NumPy's pad_mode (end and constant values 0; the statistic
 * modes take rowstat[r], the statistic of row r), then
 * real(ifft(fft(row) * ifftshift(|W|))) cropped to [pad, pad + ncol).
 * One row per transform: a row's result depends on that row alone, bit for
 * bit (equal rows give equal results).
 *
 *   spectrum  complex128 [fft_len]: transform of the filter kernel laid on
 *             the length-fft_len circle at the lags the crop uses, / fft_len
 *   twiddle   complex128 [fft_len]: exp(-2 pi i t / fft_len)
 *   fft_len   atb_filter_rows64_length(ncol, pad): ncol + 2 pad when it has
 *             no prime factor above 13, else a 7-smooth length of at least
 *             2 ncol + 2 pad - 1; at most 7168
 * src and dst may be the same rows.
 */
int atb_filter_rows64_length(int ncol, int pad);
int atb_filter_rows64(const double *src, int64_t src_row_stride, int nrows,
                      int ncol, int pad, int pad_mode,
                      const double *rowstat, const void *spectrum,
                      const void *twiddle, int fft_len, double *dst,
                      int64_t dst_row_stride, void *stream);

/*
 * Row maxima of the "autocorrelation" metric of the vertical centre search
 * (__calculate_autocorrelation_coefficient, algotom/rec/vertrec.py:
 * 1255-1261, mean(max(|ifft(|fft(row)|^2)|, axis=1))): out[r] = the largest
 * |circular autocorrelation| of float32 row r over all lags, in FP64; the
 * caller takes the mean of the rows of each image.
 *
 *   twiddle  complex128 [fft_len]: exp(-2 pi i t / fft_len)
 *   fft_len  atb_autocorr_length(ncol): ncol when it has no prime factor
 *            above 13, else a 7-smooth length of at least 2 ncol - 1 (the
 *            linear autocorrelation, folded onto the circle); at most 7168
 *   out      device float64 [nrows]
 */
int atb_autocorr_length(int ncol);
int atb_autocorr_rowmax(const float *src, int64_t src_row_stride, int nrows,
                        int ncol, const void *twiddle, int fft_len,
                        double *out, void *stream);

/* ---------------------------------------------------------------------- */
/* Total variation of the sparse-view model-based reconstruction          */
/* ---------------------------------------------------------------------- */

/*
 * Smoothed isotropic total variation of a float32 [ny][nx] image (rows
 * row_stride apart), TV = sum over i < ny-1, j < nx-1 of
 * sqrt(dx^2 + dy^2 + eps) with dx = x[i][j+1] - x[i][j],
 * dy = x[i+1][j] - x[i][j], and its gradient.  No counterpart in the
 * reference (it has no iterative reconstruction on this path); it is the
 * regulariser of the least-squares + TV descent that drives the
 * differentiable back-projection.
 *
 * atb_tv_value: *out (device float32) = TV, summed in FP64 in a fixed
 *   order; workspace: atb_tv_workspace() bytes of device memory.
 * atb_tv_grad: grad = (weight * *scale) dTV/dx (scale a device float32, or
 *   null for 1), added to grad when accumulate is nonzero.
 */
int64_t atb_tv_workspace(void);
int atb_tv_value(const float *img, int64_t row_stride, int ny, int nx,
                 double eps, void *workspace, int64_t workspace_bytes,
                 float *out, void *stream);
int atb_tv_grad(const float *img, int64_t row_stride, int ny, int nx,
                double eps, const float *scale, float weight, float *grad,
                int64_t grad_row_stride, int accumulate, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ALGOTOM_B200_H */
