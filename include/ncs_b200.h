/*
 * ncs_b200.h -- C ABI of libncs_b200.so, the B200 (sm_100a) implementation of
 * the NCS per-tile L-BFGS denoising path.
 *
 * Plain C types only: pointers, sizes and a POD parameter struct.  Device
 * buffers are raw CUDA device pointers (e.g. torch.Tensor.data_ptr()); the
 * caller owns them.  `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Every call returns NCSB_OK (0) or a negative
 * NCSB_E* code and never aborts; ncsb_last_error() describes the last failure
 * on a handle.  One handle must not be used by two host threads at once, and
 * two launches on one handle must not overlap on the GPU (they share the
 * handle's work-queue counter).
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

/* Tile geometry is fixed: 16x16 tiles, 14x14 interiors, stride 14. */
#define NCSB_TILE 16

typedef struct {
    double alpha;      /* NCS alpha (ncs.c:352, ncs.cu:959) */
    int32_t max_iters; /* L-BFGS iteration cap (ncs.cu MAXITERS = 200) */
    int32_t m;         /* history pairs, 1..8, at most 4 in the spectral form (ncs.cu M = 8;
                          libLBFGS m = 6; default 2: NCS tiles need the same number of
                          iterations for every m measured, 1..8 in the plain form and
                          1..4 in the spectral one, and fewer pairs cost less) */
    double epsilon;    /* stop when ||g|| <= epsilon * max(1, ||u||)
                          (ncs.cu EPSILON = 1e-4; libLBFGS epsilon = 1e-5) */
    double c1;         /* Armijo constant (ncs.cu C_1 = 1e-4) */
    double min_step;   /* line search gives up below this step (ncs.cu MIN_STEP 1e-6) */
    int32_t mode;      /* NCSB_MODE_* */
    int32_t ctas_per_sm; /* persistent grid: resident CTAs per SM, 0 = occupancy max */
} ncsb_params;

typedef struct ncsb_handle ncsb_handle;

/* Fill *p with the defaults: alpha 0.2, max_iters 200, m 2, epsilon 1e-5,
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
 * Tile-level solve with the reference kernel's data layout: data_in and
 * gamma_in are [n_tiles][16][16] FP32 (gamma per tile, ncs.cu:931),
 * data_out [n_tiles][16][16]; iters / status / cost / evals optional [n_tiles].
 * u0 (optional, [n_tiles][16][16]) replaces the start u0 = data_in.
 */
int ncsb_solve_tiles(ncsb_handle *h, const float *data_in, const float *gamma_in,
                     const float *u0, int64_t n_tiles, float *data_out, int32_t *iters,
                     int32_t *status, double *cost, int32_t *evals, void *stream);

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
 * geometry) and should come before any stream capture.  Every call shares the
 * array and re-initialises it on its own stream (mask table copy, counter
 * reset) before its launch, so calls that overlap on the GPU -- on two
 * streams or from two host threads -- race and must be serialised by the
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
