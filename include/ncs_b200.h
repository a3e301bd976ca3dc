/*
 * ncs_b200.h -- C ABI of libncs_b200.so, the B200 (sm_100a) implementation of
 * the NCS per-tile L-BFGS denoising path.
 *
 * Plain C types only: pointers, sizes and a POD parameter struct.  Device
 * buffers are raw CUDA device pointers (e.g. torch.Tensor.data_ptr()); the
 * caller owns them.  `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Every call returns NCSB_OK (0) or a negative
 * NCSB_E* code and never aborts; ncsb_last_error() describes the last failure
 * on a handle.  A call for 0 frames (or 0 tiles) checks its shape and
 * parameters and does nothing; its data buffers may then be null (an empty
 * tensor's data_ptr() is 0).  One handle must not be used by two host
 * threads at once, and two launches on one handle must not overlap on the
 * GPU (they share the handle's work-queue counter).
 *
 * Reference interfaces replaced (paths in the HuanglabPurdue/NCS tree):
 *   ncsb_reduce_noise  <- C   ncsReduceNoise(double*, double*, double*, double*,
 *                               double, int, int, int)  clib/pyCNCS/ncs.c:41-48,
 *                               clib/pyCNCS/ncs.h:42
 *                         Py  pyCUDANCS.ncs.NCSCUDA.reduceNoise
 *                               cuda/pyCUDANCS/ncs.py:35-173 (host tiling,
 *                               launch, stitch -- all on the device here)
 *   ncsb_solve_tiles   <- CUDA kernel ncsReduceNoise(float4 *data_in,
 *                               float4 *g_gamma, float4 *otf_mask, float4 *data_out,
 *                               int *g_iterations, int *g_status, float alpha)
 *                               cuda/ncs.cu:873-879 (tiles in, tiles out)
 *   ncsb_set_otf_mask  <- ncsSRSetOTFMask clib/pyCNCS/ncs.c:502-510 and
 *                               NCSCUDA.setOTFMask cuda/pyCUDANCS/ncs.py:183-197
 *   ncsb_create / ncsb_destroy <- ncsSRInitialize / ncsSRCleanup
 *                               clib/pyCNCS/ncs.c:394-446, :307-327
 */
#ifndef NCS_B200_H
#define NCS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes of the ABI. */
#define NCSB_OK 0
#define NCSB_EINVAL (-1)   /* bad argument (null pointer, size, parameter) */
#define NCSB_ECUDA (-2)    /* a CUDA runtime call failed */
#define NCSB_ENOMASK (-3)  /* ncsb_set_otf_mask() has not been called */
#define NCSB_ESIZE (-4)    /* image smaller than a tile interior on an axis */
#define NCSB_ESCRATCH (-5) /* request needs more than the static scratch holds */

/* Capacity of the static device scratch of ncsb_reduce_noise_noalloc. */
#define NCSB_NOALLOC_SCRATCH_BYTES 4096

/* Per-tile solver status (same values as cuda/ncs.cu:61-67). */
#define NCSB_SUCCESS 0
#define NCSB_UNSTARTED (-1)
#define NCSB_REACHED_MAXITERS (-2)
#define NCSB_INCREASING_GRADIENT (-3)
#define NCSB_MINIMUM_STEP (-4)
#define NCSB_REACHED_MAXPRECISION (-5)

/* Solver forms. */
#define NCSB_MODE_PLAIN 0     /* FP32 SIMT, one warp per tile, in-register/smem FFT */
#define NCSB_MODE_PLAIN_WG 1  /* FP32 SIMT, one warp group per tile (comparison form) */
#define NCSB_MODE_SPECTRAL 2  /* FP32 SIMT, one warp per tile, L-BFGS with the spectral
                                 initial inverse Hessian (lambda I + 2 alpha Q)^-1; m <= 4 */
/* Tensor-core forms: the spectral form's algorithm with every 16x16 transform
   of the noise term Q u = (1/256) F^H diag(M^2) F u (and of the initial
   inverse Hessian) done as four tcgen05 GEMMs over 8 tiles at a time, FP32
   accumulation; m = 1.  They replace the FFT noise term and its gradient of
   cuda/ncs.cu:743-817 and clib/pyCNCS/ncs.c:220-299.  The per-tile cost they
   report is the solver's running value (v = 2 alpha Q u kept by updates). */
#define NCSB_MODE_TC_TF32 3   /* TF32 operands */
#define NCSB_MODE_TC_BF16X3 4 /* three-way BF16 split: hi*hi + lo*hi + hi*lo */

/* Tile geometry is fixed: 16x16 tiles, 14x14 interiors, stride 14. */
#define NCSB_TILE 16

typedef struct {
    double alpha;      /* NCS alpha (ncs.c:352, ncs.cu:959) */
    int32_t max_iters; /* L-BFGS iteration cap (ncs.cu MAXITERS = 200) */
    int32_t m;         /* history pairs, 1..8, at most 4 in the spectral form (ncs.cu M = 8;
                          libLBFGS m = 6; default 1: NCS tiles need the same number of
                          iterations for every m measured, 1..8 in the plain form and
                          1..4 in the spectral one, and fewer pairs cost less -- the
                          spectral solve measured about 6 % slower at m = 2 than at
                          m = 1) */
    double epsilon;    /* stop when ||g|| <= epsilon * max(1, ||u||)
                          (ncs.cu EPSILON = 1e-4; libLBFGS epsilon = 1e-5) */
    double c1;         /* Armijo constant (ncs.cu C_1 = 1e-4) */
    double min_step;   /* line search gives up below this step (ncs.cu MIN_STEP 1e-6) */
    int32_t mode;      /* NCSB_MODE_* */
    int32_t ctas_per_sm; /* persistent grid: resident CTAs per SM, 0 = occupancy max */
} ncsb_params;

typedef struct ncsb_handle ncsb_handle;

/* Fill *p with the defaults: alpha 0.2, max_iters 200, m 1, epsilon 1e-5,
 * c1 1e-4, min_step 1e-6, spectral form, auto grid. */
void ncsb_default_params(ncsb_params *p);

/* Create a handle on the current CUDA device; allocates its small device
 * workspace (queue counter, mask tables). */
int ncsb_create(ncsb_handle **out, const ncsb_params *p);
int ncsb_set_params(ncsb_handle *h, const ncsb_params *p);
int ncsb_destroy(ncsb_handle *h);
const char *ncsb_last_error(const ncsb_handle *h);

/* OTF mask, 16x16 row-major FP32 in HOST memory, already fftshifted so that
 * DC is at [0][0] (the convention of ncs.c and cuda/ncs.cu).  The handle
 * squares it and builds the device tables.  Symmetry is the caller's check
 * (the Python layer mirrors checkOTFMask, ncs_c.py:239-247). */
int ncsb_set_otf_mask(ncsb_handle *h, const float *mask_shifted_host);

/* Number of 16x16 tiles an n_frames x height x width stack is cut into:
 * per axis the length of range(0, n+2, 14) with the last origin clamped to
 * n+2-16 (ncs.c:71-86); 0 and NCSB_ESIZE if an axis is shorter than 14. */
int ncsb_num_tiles(int n_frames, int height, int width, int64_t *n_tiles);

/*
 * Whole-stack NCS on the device.  images: [n_frames][height][width] FP32
 * photo-electrons (non-positive values already replaced by a small positive
 * value, as ncs.c:4-8 requires); gamma: [height][width] read-noise variance /
 * gain^2 shared by all frames when gamma_per_frame == 0, else
 * [n_frames][height][width].  out: [n_frames][height][width].  Segmentation
 * (1-px edge-replicated halo) and stitching (later tiles win on overlaps,
 * ncs.c:121-130) happen inside the kernel.  tile_iters / tile_status /
 * tile_cost (final FP64 cost) are optional per-tile outputs of length
 * ncsb_num_tiles(), in (frame, tile-row, tile-col) order; pass NULL to skip.
 * tile_evals (optional) counts cost evaluations per tile: the initial one
 * plus one per line-search trial.
 * height and width must be >= 14.
 */
int ncsb_reduce_noise(ncsb_handle *h, const float *images, int n_frames, int height, int width,
                      const float *gamma, int gamma_per_frame, float *out, int32_t *tile_iters,
                      int32_t *tile_status, double *tile_cost, int32_t *tile_evals,
                      void *stream);

/*
 * ncsb_reduce_noise from and to HOST memory, the form of the reference's
 * Python entries (cuda/pyCUDANCS/ncs.py:137-147 copies the tiles to the
 * device, launches, and copies the result back; clib/pyCNCS/ncs_c.py:250-276
 * works on host arrays).  images, gamma (shared or per frame, as in
 * ncsb_reduce_noise) and out are host pointers; page-locked memory lets the
 * copies overlap the solve.  The stack is cut into chunks of chunk_frames
 * frames (<= 0: n_frames / 40, at most 64 MB); chunk i is copied in, solved
 * and copied out on
 * the handle's stream i % n_streams (<= 0: 4; at most 8), each stream with its own
 * device buffers and work counter, so one chunk's copies overlap other
 * chunks' copies and solves.  The streams start after the work already
 * queued on `stream`, and `stream` waits for them.  The call returns once
 * `out` holds the result.  The handle's streams, events and buffers are
 * created on the first call and kept until ncsb_destroy; calls on one
 * handle must not overlap.  Results equal ncsb_reduce_noise bit for bit.
 */
int ncsb_reduce_noise_host(ncsb_handle *h, const float *images, int n_frames, int height,
                           int width, const float *gamma, int gamma_per_frame, float *out,
                           int chunk_frames, int n_streams, void *stream);

/*
 * Tile-level solve with the reference kernel's data layout: data_in and
 * gamma_in are [n_tiles][16][16] FP32 (gamma per tile, ncs.cu:931),
 * data_out [n_tiles][16][16]; iters / status / cost / evals optional [n_tiles].
 * u0 (optional, [n_tiles][16][16]) replaces the start u0 = data_in; in the
 * spectral form a tile whose u0 has a higher cost than data_in starts at
 * data_in (as in ncsb_reduce_noise_start).
 */
int ncsb_solve_tiles(ncsb_handle *h, const float *data_in, const float *gamma_in,
                     const float *u0, int64_t n_tiles, float *data_out, int32_t *iters,
                     int32_t *status, double *cost, int32_t *evals, void *stream);

/*
 * ncsb_reduce_noise from a proposed start (the learned warm start; no
 * counterpart in the reference, whose solve always starts at u = d,
 * clib/pyCNCS/ncs.c:548-551, cuda/ncs.cu:933).  u0_tiles: [ncsb_num_tiles()][16][16] FP32,
 * one proposal per tile in (frame, tile-row, tile-col) order, halo included,
 * as ncsb_net_infer_stack writes it.  Each tile starts at its proposal unless
 * the proposal's cost is higher than that of the photon image, in which case
 * it starts at u = d exactly as ncsb_reduce_noise does; the stopping rule is
 * unchanged.  tile_start (optional, [n_tiles]) receives 0 where the proposal
 * was used and 1 where the tile fell back to the photon image.  Spectral form
 * only (NCSB_EINVAL otherwise); other arguments as ncsb_reduce_noise.
 */
int ncsb_reduce_noise_start(ncsb_handle *h, const float *images, int n_frames, int height,
                            int width, const float *gamma, int gamma_per_frame,
                            const float *u0_tiles, float *out, int32_t *tile_iters,
                            int32_t *tile_status, double *tile_cost, int32_t *tile_evals,
                            int32_t *tile_start, void *stream);

/* ---- raw camera frames: the preprocessing prologue on the device -----------
 * The reference converts ADU to photo-electrons on the host before the solve
 * (python3-6/pyNCS/denoisetools.py:222-224, python3-6/NCSdemo_experiment.py:47-49:
 * d = (ADU - offset) / gain, d <= 0 -> 1e-6; gamma = var / gain^2,
 * denoisetools.py:266), and for cameras with several gain amplifiers picks
 * each pixel's gain and variance maps by its ADU level (matlab/genmaps.m:29-62:
 * level 0 below levels[0], level k for levels[k-1] <= ADU < levels[k], the
 * last level above the last threshold).  Here one device pass does this per
 * pixel into a buffer the handle owns, and the solve reads it: the frames
 * never return to the host between conversion and solve. */
typedef struct {
    const float *offset;    /* device [height][width], ADU */
    const float *gain;      /* device [n_levels][height][width], ADU per photo-electron (> 0) */
    const float *variance;  /* device [n_levels][height][width], ADU^2 */
    int32_t n_levels;       /* 1..4 gain / variance map pairs */
    float levels[3];        /* ascending ADU thresholds between the pairs (n_levels - 1 used) */
} ncsb_calibration;

/* ncsb_reduce_noise on raw ADU frames adu [n_frames][height][width] with the
 * camera calibration `cal` (host struct of device pointers).  out is in
 * photo-electrons, as ncsb_reduce_noise's.  Any solver form.  The handle
 * allocates (and keeps, growing it when needed) a device buffer of
 * n_frames x height x width floats, twice that with several map pairs. */
int ncsb_reduce_noise_adu(ncsb_handle *h, const float *adu, int n_frames, int height, int width,
                          const ncsb_calibration *cal, float *out, int32_t *tile_iters,
                          int32_t *tile_status, double *tile_cost, int32_t *tile_evals,
                          void *stream);

/* Element types of raw frames: FP32 counts, or the unsigned integers cameras
 * store (the reference's experimental stack, python3-6/EB300004.mat 'ims',
 * is 8-bit; its script converts the counts in float64,
 * python3-6/NCSdemo_experiment.py:47-49).  Integer counts convert to FP32
 * exactly, so an integer stack gives the same result, bit for bit, as the
 * same counts passed as FP32. */
#define NCSB_ADU_F32 0
#define NCSB_ADU_U16 1
#define NCSB_ADU_U8 2

/* ncsb_reduce_noise_adu on device frames of element type adu_type
 * (NCSB_ADU_*); NCSB_EINVAL for another type. */
int ncsb_reduce_noise_adu_typed(ncsb_handle *h, const void *adu, int adu_type, int n_frames,
                                int height, int width, const ncsb_calibration *cal, float *out,
                                int32_t *tile_iters, int32_t *tile_status, double *tile_cost,
                                int32_t *tile_evals, void *stream);

/* Raw frames in HOST memory (element type adu_type) to photo-electron
 * results in host memory, pipelined like ncsb_reduce_noise_host: chunk i of
 * chunk_frames frames (<= 0: T / 40, at most 64 MB of FP32) is copied in as
 * raw counts, converted, solved and copied out on stream i % n_streams
 * (<= 0: 4).  The calibration maps of `cal` are device pointers; adu and out
 * should be page-locked for the copies to overlap.  Returns after the last
 * copy out; out equals ncsb_reduce_noise_adu_typed's result bit for bit. */
int ncsb_reduce_noise_adu_host(ncsb_handle *h, const void *adu, int adu_type, int n_frames,
                               int height, int width, const ncsb_calibration *cal, float *out,
                               int chunk_frames, int n_streams, void *stream);

/* ---- OTF masks from optics parameters, built on the device ---------------
 * genfilter of the reference (python3-6/pyNCS/denoisetools.py:227-261 with
 * genkspace :96-101): a raised-cosine high-pass of the radial frequency
 * |k| = sqrt(X^2 + Y^2) / (16 pixel_size), X, Y = -8..7, for the types
 * pureN, adjustable (w, h) and OTFweighted; plus INCOHERENT, 1 - the
 * circular-pupil incoherent OTF inside the cutoff 2 NA / lambda (1 outside),
 * the mask of the synthetic workloads.  Lengths in one unit (e.g. um). */
#define NCSB_MASK_OTFWEIGHTED 0
#define NCSB_MASK_PUREN 1
#define NCSB_MASK_ADJUSTABLE 2
#define NCSB_MASK_INCOHERENT 3

typedef struct {
    int32_t type;        /* NCSB_MASK_* */
    double pixel_size;   /* sample spacing */
    double na;           /* numerical aperture */
    double wavelength;   /* emission wavelength */
    double w, h;         /* adjustable type only: 0 < w, 0 < h < 1 (reference defaults 1, 0.7) */
} ncsb_optics;

/* n centred 16x16 masks (DC at [8][8], the reference's orientation) written
 * to masks_centred (device, [n][16][16] FP32), computed in FP64 on the
 * device.  NCSB_EINVAL for an unknown type or non-positive parameters. */
int ncsb_genfilter(const ncsb_optics *optics, int n, float *masks_centred, void *stream);

/* genpsfparam of the reference (python3-6/pyNCS/denoisetools.py:103-115) on
 * the device, FP64: pupil = |k| on the centred R x R grid (genkspace), 0 above
 * NA / lambda; PSF = |fftshift(fft2(pupil))|^2 normalised to unit sum;
 * OTF = |fftshift(ifft2(PSF))| normalised to unit maximum.  Outputs are device
 * [R][R] FP32 arrays, any of them NULL to skip; 2 <= R <= 1024. */
int ncsb_genpsfparam(int R, double pixel_size, double na, double wavelength, float *psf,
                     float *pupil, float *otf, void *stream);

/* ---- simulator: synthetic sCMOS stacks generated on the device ------------
 * Replaces the reference's host-side simulation loops (python3-6/pyNCS/
 * denoisetools.py:118-186 genidealimage / SRhist, :205-225 addnoise /
 * gendatastack).  Random numbers come from Philox4x32-10 keyed by `seed` and
 * addressed by (pixel, frame, draw), so results do not depend on the launch. */

/* ideal [height][width] = background + sum over emitters of photons x the
 * pixel-integrated Gaussian PSF (sigma_px, footprint |floor(x_e) - x| <= half,
 * half <= 16).  emitters_sorted: device [n][3] FP32 (x along width, y along
 * height, photons; pixel i spans [i, i+1)), sorted by 8 x 8-pixel cell
 * (cell = clamp(floor(y)/8) * ceil(width/8) + clamp(floor(x)/8));
 * cell_start: device [ncells + 1] int32 offsets into the sorted list. */
int ncsb_sim_render(const float *emitters_sorted, const int *cell_start, int height, int width,
                    double sigma_px, int half, float background, float *ideal, void *stream);

/* n_frames independent camera frames of one ideal image: n ~ Poisson(ideal),
 * ADU = n gain + sqrt(variance) N(0,1) + offset (addnoise), and/or the
 * photo-electrons (ADU - offset) / gain with values <= 0 set to 1e-6
 * (gendatastack).  Maps [height][width]; adu and photo_electrons
 * [n_frames][height][width] (either may be NULL, not both). */
int ncsb_sim_camera(const float *ideal, int n_frames, int height, int width, const float *offset,
                    const float *gain, const float *variance, uint64_t seed, float *adu,
                    float *photo_electrons, void *stream);

/* The reference simulator's ideal image (genidealimage,
 * python3-6/pyNCS/denoisetools.py:150-186): n positions (xs -> row, ys ->
 * column) already on the fine grid of (R zoom)^2 pixels, their occupancy,
 * the 'same' convolution with the ksz x ksz PSF kernel (the centre of
 * genpsfparam's PSF), |.|, and zoom x zoom binning divided by zoom, into
 * out [R][R] (zoom 1: transposed, as the reference).  fine: device scratch
 * of (R zoom)^2 floats, overwritten. */
int ncsb_sim_ideal_image(const float *xs, const float *ys, int n, int R, int zoom,
                         const float *kernel, int ksz, float *fine, float *out, void *stream);

/* The generator's uniform deviates in (0, 1) for counters (i, frame, 0, 0),
 * i < n (for statistical tests of the generator). */
int ncsb_sim_uniforms(int64_t n, uint32_t frame, uint64_t seed, float *out, void *stream);

/* ---- normalised single-pixel variant -------------------------------------
 * The reference's "matlab - single pixel with normalization" package: every
 * pixel is its own 3 x 3 segment (the pixel and its 8 neighbours, replicate-
 * padded; segpadimg.m with Rs = 1) minimising
 *   f(u) = 2/9 sum[u - (d + gamma) log(u + gamma)]
 *          + alpha sum((|fftshift(fft2(u))| / 3 .* mask)^2) / sum(u)
 * (calcost.m:38-56) from u = d; the segment centre is kept (stitchpadimg.m)
 * and values < 0 become 1e-6 (reducenoise.m).  One thread per pixel, FP64
 * BFGS with a backtracking line search; stops when ||g||_inf <= tolerance *
 * max(1, ||g_0||_inf) or after max_iters iterations (the reference's
 * iterationN, 15 in its demos).  mask3_centred: 3 x 3 host array, centred
 * (the reference's default is genfilter(3, pixel, 2 NA, lambda)).  images,
 * gamma (shared [height][width] or per frame) and out as ncsb_reduce_noise;
 * px_iters / px_status / px_cost optional per pixel ([n_frames][height][width],
 * status codes as the main solver, cost the final FP64 f).  Allocates
 * nothing and needs no handle. */
int ncsb_reduce_noise_normalized(const float *images, int n_frames, int height, int width,
                                 const float *gamma, int gamma_per_frame,
                                 const float *mask3_centred, double alpha, int max_iters,
                                 double tolerance, float *out, int32_t *px_iters,
                                 int32_t *px_status, double *px_cost, void *stream);

/* ---- batched launch: many stacks, one persistent queue -------------------
 * No counterpart in the reference, which processes one stack per call with
 * one alpha and one mask (cuda/pyCUDANCS/ncs.py:35-173).  Here several stacks
 * -- each with its own shape, alpha and OTF mask -- are solved by one launch
 * whose work queue spans all their tiles, so small stacks do not leave the GPU
 * idle and a whole acquisition session is one kernel.  Spectral form only. */
typedef struct {
    const float *images;      /* device [n_frames][height][width] photo-electrons */
    const float *gamma;       /* device [height][width] (gamma_per_frame == 0) or
                                 [n_frames][height][width] */
    float *out;               /* device [n_frames][height][width] */
    int32_t n_frames, height, width, gamma_per_frame;
    double alpha;             /* this stack's alpha */
    float mask_shifted[256];  /* this stack's 16x16 OTF mask, DC at [0][0] (host values) */
    int32_t mask_from_optics; /* nonzero: ignore mask_shifted, build the mask from optics
                                 on the device */
    ncsb_optics optics;
} ncsb_stack;

#define NCSB_MAX_STACKS 65536

/* Upload the descriptors of n_stacks stacks (1..NCSB_MAX_STACKS) to the
 * handle: validation as ncsb_reduce_noise per stack (NCSB_ESIZE for frames
 * under 14 x 14), per-stack mask tables, tile ranges.  Synchronous; allocates
 * only when n_stacks exceeds the largest batch the handle has held.  The
 * device buffers named in the descriptors must stay valid while the batch is
 * launched. */
int ncsb_batch_set(ncsb_handle *h, const ncsb_stack *stacks, int n_stacks);

/* Total tiles of the current batch: the sum of ncsb_num_tiles() over its
 * stacks, in stack order (the order of the per-tile outputs). */
int ncsb_batch_num_tiles(const ncsb_handle *h, int64_t *n_tiles);

/* Solve every tile of the current batch in one launch on `stream`: a counter
 * reset and one kernel, nothing else, so the call can be captured into a CUDA
 * graph and replayed (ncsb_batch_set must happen before the capture).
 * u0_tiles (optional, [n_tiles][16][16]) gives proposed starts as in
 * ncsb_reduce_noise_start, tile_start (optional) receives the fallback flags;
 * tile_iters / tile_status / tile_cost / tile_evals are optional [n_tiles]. */
int ncsb_batch_reduce_noise(ncsb_handle *h, const float *u0_tiles, int32_t *tile_iters,
                            int32_t *tile_status, double *tile_cost, int32_t *tile_evals,
                            int32_t *tile_start, void *stream);

/* ---- learned warm start: a 4-layer 3x3 convolutional network ------------
 * Maps each tile's photon image d and gamma map to a proposed start.  Input
 * features per tile: x0 = (d - mu) / s, x1 = sqrt(max(d, 0) + gamma) / s with
 * mu, s = mean and standard deviation + 1 of the tile's d; layers 2->32->32->32->1
 * channels, 3x3 kernels with zero padding, ReLU after the first three; the
 * proposal is u0 = d + s y.  No counterpart in the reference.
 *
 * Tensors are FP32 device buffers: activations [n][channels][16][16]; weights
 * of a layer stored as wt[cin][3*ky + kx][cout] (ky, kx the kernel offsets
 * -1..1 shifted by one), bias [cout].  The packed parameter vector of the
 * whole network holds w1, b1, w2, b2, w3, b3, w4, b4 in that order
 * (ncsb_net_param_count() floats).  All calls are asynchronous on `stream`. */
int ncsb_net_param_count(void);

/* y = conv3x3(x) + b (ReLU if relu), for (cin, cout) in {(2,32), (32,32),
 * (32,1), (1,32)}; b may be NULL (zero bias).  One 16x16 image per tile. */
int ncsb_net_conv_fwd(const float *x, const float *wt, const float *b, float *y, int n_tiles,
                      int cin, int cout, int relu, void *stream);

/* Weight and bias gradients of conv3x3, ACCUMULATED into dwt [cin][9][cout]
 * and db [cout]: dwt += sum_tiles,pixels x (*) dy, db += sum dy.
 * (cin, cout) in {(2,32), (32,32), (32,1)}. */
int ncsb_net_conv_wgrad(const float *x, const float *dy, float *dwt, float *db, int n_tiles,
                        int cin, int cout, void *stream);

/* Weights of the input-gradient convolution: wf[cout][8 - tap][cin] =
 * wt[cin][tap][cout], so that ncsb_net_conv_fwd(dy, wf, NULL, dx, n, cout,
 * cin, 0) gives dx = conv3x3^T(dy). */
int ncsb_net_flip(const float *wt, float *wf, int cin, int cout, void *stream);

/* g[i] = 0 where act[i] <= 0 (ReLU backward through the layer output act). */
int ncsb_net_relu_bwd(float *g, const float *act, int64_t n, void *stream);

/* Mean squared error: g = 2 (y - t) / n, and loss[0] += mean((y - t)^2)
 * (loss must be zeroed by the caller). */
int ncsb_net_mse_grad(const float *y, const float *t, float *g, float *loss, int64_t n,
                      void *stream);

/* One Adam step (bias-corrected, step >= 1) over n parameters. */
int ncsb_net_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                  float b2, float eps, int step, void *stream);

/* Network input features x [n][2][16][16] and per-tile (mu, s) scale [n][2]
 * from tiles d, gamma [n][16][16]. */
int ncsb_net_features(const float *d, const float *gamma, float *x, float *scale, int n_tiles,
                      void *stream);

/* Whole-network inference straight from a stack: cuts each tile (the
 * solvers' segmentation) and writes the proposal u0_tiles
 * [ncsb_num_tiles()][16][16] for ncsb_reduce_noise_start.  Proposals are
 * kept feasible: u0 + gamma >= 0.05 max(d + gamma, 1e-3). */
int ncsb_net_infer_stack(const float *params, const float *images, int n_frames, int height,
                         int width, const float *gamma, int gamma_per_frame, float *u0_tiles,
                         void *stream);

/* The same inference over the handle's current batch (ncsb_batch_set):
 * u0_tiles [ncsb_batch_num_tiles()][16][16] in the batch's tile order. */
int ncsb_net_infer_batch(const float *params, const ncsb_handle *h, float *u0_tiles,
                         void *stream);

/* ncsb_net_infer_stack on the tensor cores (tcgen05): BF16 weights and
 * activations, FP32 accumulation in tensor memory; the layers as implicit
 * GEMMs over the zero-bordered 18 x 18 plane (M = 128, N = 32, K = 16).
 * Results differ from the FP32 kernel by BF16 rounding (about 1e-2 of the
 * tile's scale s at most).  status (optional, device int32): set to 1 if a
 * wait for the tensor cores timed out (the kernel then ends early). */
int ncsb_net_infer_stack_tc(const float *params, const float *images, int n_frames, int height,
                            int width, const float *gamma, int gamma_per_frame, float *u0_tiles,
                            int32_t *status, void *stream);

/* The tensor-core inference over the handle's current batch (ncsb_batch_set):
 * u0_tiles [ncsb_batch_num_tiles()][16][16] in the batch's tile order. */
int ncsb_net_infer_batch_tc(const float *params, const ncsb_handle *h, float *u0_tiles,
                            int32_t *status, void *stream);

/* The tensor-core inference on tiles d, gamma [n][16][16] -> u0 [n][16][16]. */
int ncsb_net_infer_tiles_tc(const float *params, const float *d, const float *gamma,
                            int64_t n_tiles, float *u0, int32_t *status, void *stream);

/* The three tensor-core inferences above with E4M3 (FP8) operands
 * (tcgen05 kind::f8f6f4, K = 32 per MMA; activations stored as three
 * column-shifted copies so that each layer is 2 M blocks x 9 taps): about
 * twice the speed of the BF16 form.  Each output channel's weights are divided
 * by (its largest |w|) / 448 before rounding, the network's input features
 * are multiplied by 8 and the hidden activations by 4 (exact powers of two;
 * values beyond E4M3's range saturate at +-448), and the epilogue undoes
 * both scales in FP32.  Proposals differ from the FP32 network's by about
 * 0.03-0.05 of the tile's scale s on average (single pixels up to about s);
 * the solve from them is unchanged in its stopping rule and fallback, and
 * takes the same iterations. */
int ncsb_net_infer_stack_tc_fp8(const float *params, const float *images, int n_frames,
                                int height, int width, const float *gamma, int gamma_per_frame,
                                float *u0_tiles, int32_t *status, void *stream);
int ncsb_net_infer_batch_tc_fp8(const float *params, const ncsb_handle *h, float *u0_tiles,
                                int32_t *status, void *stream);
int ncsb_net_infer_tiles_tc_fp8(const float *params, const float *d, const float *gamma,
                                int64_t n_tiles, float *u0, int32_t *status, void *stream);

/* The same inference on tiles d, gamma [n][16][16] -> u0 [n][16][16]. */
int ncsb_net_infer_tiles(const float *params, const float *d, const float *gamma, int64_t n_tiles,
                         float *u0, void *stream);

/*
 * ncsb_reduce_noise without a handle and without allocating device memory.
 * No counterpart in the reference: it exists for callers that may not call
 * cudaMalloc while they run -- a plug-in in an acquisition or image-server
 * process whose host application owns the GPU memory budget through its own
 * pool, or a real-time pipeline that forbids device allocation after start-up
 * because cudaMalloc can synchronise the device and stall the camera stream.
 * Such callers cannot use ncsb_create, which allocates the work counter and
 * the mask table.
 *
 * Same arguments and results as ncsb_reduce_noise, plus the solver
 * parameters and the 16x16 shifted OTF mask (host memory) that a handle would
 * hold.  The work counter and the mask table live instead in one file-scope
 * __device__ array of NCSB_NOALLOC_SCRATCH_BYTES (4 KiB), held by every GPU
 * that loads the library until the process exits; this call uses 1280 bytes
 * of it whatever the stack size, and a request that would need more than the
 * capacity is rejected with NCSB_ESCRATCH.  The call allocates nothing: no
 * cudaMalloc, cudaFree or allocating library routine.
 *
 * The first call on a device does a one-time set-up (it looks up the
 * array's device address with cudaGetSymbolAddress and caches the launch
 * geometry) and should come before any stream capture; the cached address is
 * kept until the process exits, so the entry must not be used across
 * cudaDeviceReset.  Every call shares the array and re-initialises it on its
 * own stream before its launch -- a one-block kernel writes the mask table,
 * passed to it by value, and resets the work counter -- so a call never waits
 * for the stream on the host, and calls that overlap on the GPU (on two
 * streams or from two host threads) race and must be serialised by the
 * caller.
 */
int ncsb_reduce_noise_noalloc(const ncsb_params *p, const float *mask_shifted_host,
                              const float *images, int n_frames, int height, int width,
                              const float *gamma, int gamma_per_frame, float *out,
                              int32_t *tile_iters, int32_t *tile_status, double *tile_cost,
                              int32_t *tile_evals, void *stream);

#ifdef __cplusplus
}
#endif

#endif
