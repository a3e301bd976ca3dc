// ncs_capi.cu -- the extern "C" ABI of libncs_b200.so (declared in
// include/ncs_b200.h).  Owns the handle: solver parameters, the device mask
// table and the work-queue counter; mirrors ncsSRInitialize / ncsSRCleanup
// (clib/pyCNCS/ncs.c:394-446, :307-327) for the device.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ncs_b200.h"
#include "ncs_internal.cuh"

namespace ncsb {
cudaError_t launch_plain(const SolveArgs& args, int grid, cudaStream_t stream);
int plain_max_ctas_per_sm();
cudaError_t launch_warp_blocks(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int warp_max_ctas_per_sm(int m, int blocks);
cudaError_t launch_spectral(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int spectral_max_ctas_per_sm(int m, int blocks, bool warm, bool batch);
cudaError_t launch_tc(const SolveArgs& args, bool bf16x3, int grid, cudaStream_t stream);
int tc_max_ctas_per_sm(bool bf16x3, bool warm);
int tc_tiles_per_cta();
namespace masks {
bool valid(const ncsb_optics& o);
cudaError_t launch_masks(const ncsb_optics* d_optics, int n, float* centred, float* lane,
                         const int* d_slot, cudaStream_t s);
}  // namespace masks
namespace net {
int launch_infer_batch(const float* params, const StackDesc* stacks, int n_stacks,
                       long long n_tiles, float* u0, cudaStream_t s);
}  // namespace net
namespace adu {
cudaError_t launch_convert(const void* adu, int adu_type, int T, int H, int W,
                           const ncsb_calibration* cal, float* d, float* gamma_frames,
                           float* gamma_map, cudaStream_t s);
cudaError_t launch_gamma_map(const ncsb_calibration* cal, long long hw, float* gamma,
                             cudaStream_t s, int num_sms);
}  // namespace adu
namespace nettc {
int launch_batch(const float* params, const StackDesc* stacks, int n_stacks, long long n_tiles,
                 float* u0, int32_t* status, bool fp8, cudaStream_t s);
}  // namespace nettc
}  // namespace ncsb

using ncsb::tiles_along;

namespace {

// State of ncsb_reduce_noise_host, created on its first call: up to
// kMaxStreams streams, each with its own chunk buffers and work counter.
// Chunk i goes to stream i % n, which copies it in, solves it and copies it
// out, so stream order alone protects each buffer and the copies of
// different streams interleave on the host link in both directions.
struct HostPipe {
    static constexpr int kMaxStreams = 8;
    int n = 0;            // streams with buffers
    size_t chunk_px = 0;  // pixels per chunk buffer
    bool per_frame = false;
    size_t gamma_px = 0;  // pixels of the shared gamma buffer
    float* d_in[kMaxStreams] = {};
    float* d_out[kMaxStreams] = {};
    float* d_gf[kMaxStreams] = {};  // per-frame gamma chunks
    float* d_gamma = nullptr;       // shared gamma map
    unsigned long long* d_queues = nullptr;  // [kMaxStreams]
    cudaStream_t st[kMaxStreams] = {};
    cudaEvent_t start = nullptr, gamma_in = nullptr, done[kMaxStreams] = {};
};

// Wait for everything queued on the pipeline's streams (before its buffers
// are freed or resized, and when a call stops early on an error).
void sync_pipe(HostPipe* q) {
    for (cudaStream_t st : q->st)
        if (st) cudaStreamSynchronize(st);
}

void free_buffers(HostPipe* q) {
    for (int b = 0; b < HostPipe::kMaxStreams; ++b) {
        cudaFree(q->d_in[b]);
        cudaFree(q->d_out[b]);
        cudaFree(q->d_gf[b]);
        q->d_in[b] = q->d_out[b] = q->d_gf[b] = nullptr;
    }
    q->n = 0;
    q->chunk_px = 0;
    q->per_frame = false;
}

void destroy_pipe(HostPipe* q) {
    if (!q) return;
    sync_pipe(q);
    free_buffers(q);
    cudaFree(q->d_gamma);
    cudaFree(q->d_queues);
    for (cudaStream_t st : q->st)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : {q->start, q->gamma_in})
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : q->done)
        if (ev) cudaEventDestroy(ev);
    delete q;
}

}  // namespace

struct ncsb_handle {
    ncsb_params p;
    int device = 0;
    int num_sms = 1;
    bool has_mask = false;
    float* d_msq = nullptr;                 // [256] M^2/256, natural [kr][kc] order
    unsigned long long* d_queue = nullptr;  // work counter
    int32_t* d_flag = nullptr;              // tensor-core forms: 1 after a wait ran out
    // batched launch (ncsb_batch_set): stack descriptors, per-stack lane-layout
    // M^2/256 tables, capacity in stacks, current count and total tiles
    ncsb::StackDesc* d_stacks = nullptr;
    float* d_mk_lane = nullptr;
    int batch_cap = 0;
    int n_stacks = 0;
    long long batch_tiles = 0;
    HostPipe* pipe = nullptr;  // ncsb_reduce_noise_host
    float* d_adu = nullptr;    // ncsb_reduce_noise_adu: converted frames, then gamma
    size_t adu_px = 0;         // capacity of d_adu in floats
    std::string err;
};

namespace {

int fail(ncsb_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(ncsb_handle* h, cudaError_t e, const char* what) {
    return fail(h, NCSB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Arguments of the raw-ADU entries; NCSB_OK when the call may go ahead (with
// n_frames == 0 it then does nothing, and adu and out may be null).
int check_adu_call(ncsb_handle* h, const void* adu, int adu_type, int n_frames, int height,
                   int width, const ncsb_calibration* cal, const float* out) {
    if (!h) return NCSB_EINVAL;
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (!cal || !cal->offset || !cal->gain || !cal->variance)
        return fail(h, NCSB_EINVAL, "null calibration map");
    if (adu_type != NCSB_ADU_F32 && adu_type != NCSB_ADU_U16 && adu_type != NCSB_ADU_U8)
        return fail(h, NCSB_EINVAL, "adu_type must be NCSB_ADU_F32, NCSB_ADU_U16 or NCSB_ADU_U8");
    if (cal->n_levels < 1 || cal->n_levels > 4)
        return fail(h, NCSB_EINVAL, "n_levels must be 1..4");
    for (int q = 0; q + 1 < cal->n_levels; ++q) {
        if (!std::isfinite(cal->levels[q]) || (q > 0 && !(cal->levels[q] > cal->levels[q - 1])))
            return fail(h, NCSB_EINVAL, "levels must be finite and ascending");
    }
    if (n_frames < 0 || height <= 0 || width <= 0) return fail(h, NCSB_EINVAL, "bad shape");
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2)
        return fail(h, NCSB_ESIZE, "frames must be at least 14 x 14");
    if (n_frames > 0 && (!adu || !out)) return fail(h, NCSB_EINVAL, "null buffer");
    return NCSB_OK;
}

int check_params(const ncsb_params* p, std::string* why) {
    if (!p) { *why = "params is NULL"; return NCSB_EINVAL; }
    if (!std::isfinite(p->alpha) || p->alpha < 0.0) { *why = "alpha must be finite and >= 0"; return NCSB_EINVAL; }
    if (p->max_iters < 0) { *why = "max_iters must be >= 0"; return NCSB_EINVAL; }
    if (p->m < 1 || p->m > ncsb::kMaxM) { *why = "m must be in 1..8"; return NCSB_EINVAL; }
    if (!(p->epsilon >= 0.0)) { *why = "epsilon must be >= 0"; return NCSB_EINVAL; }
    if (!(p->c1 > 0.0 && p->c1 < 1.0)) { *why = "c1 must be in (0, 1)"; return NCSB_EINVAL; }
    if (!(p->min_step > 0.0)) { *why = "min_step must be > 0"; return NCSB_EINVAL; }
    if (p->mode < NCSB_MODE_PLAIN || p->mode > NCSB_MODE_TC_BF16X3) { *why = "unsupported mode"; return NCSB_EINVAL; }
    if (p->ctas_per_sm < 0) { *why = "ctas_per_sm must be >= 0"; return NCSB_EINVAL; }
    return NCSB_OK;
}

// Symmetrised M^2/256 in natural order [kr][kc] from a shifted 16x16 mask.
// For real u the noise term only sees the symmetric part of M^2
// (|U_k| = |U_-k|), and the kernels' real-output inverse transforms rely on
// it; a mask passing checkOTFMask is unchanged.
bool build_msq(const float* mask, float tab[256]) {
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 16; ++j) {
            const double a = mask[i * 16 + j], b = mask[((16 - i) & 15) * 16 + ((16 - j) & 15)];
            if (!std::isfinite(a)) return false;
            tab[i * 16 + j] = (float)(0.5 * (a * a + b * b) / 256.0);
        }
    return true;
}

int bitrev3_host(int i) { return ((i & 1) << 2) | (i & 2) | ((i & 4) >> 2); }

// The spectral kernel's lane layout of the table: lane L holds, at positions
// 8 L .. 8 L + 7, the values of its 8 spectral bins (ncs_spectral.cu).
void lane_layout(const float nat[256], float* out) {
    for (int idx = 0; idx < 256; ++idx) {
        const int L = idx >> 3, i = idx & 7;
        out[idx] = nat[(2 * bitrev3_host(i) + (L & 1)) * 16 + (L >> 1)];
    }
}

// queue: the work counter of this launch (default: the handle's own)
int launch(ncsb_handle* h, ncsb::SolveArgs& a, cudaStream_t s, unsigned long long* queue = nullptr) {
    if (!queue) queue = h->d_queue;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemsetAsync(queue)");
    a.queue = queue;
    a.msq = h->d_msq;
    a.alpha = (float)h->p.alpha;
    a.eps = (float)h->p.epsilon;
    a.c1 = (float)h->p.c1;
    a.min_step = (float)h->p.min_step;
    a.max_iters = h->p.max_iters;
    a.m = h->p.m;
    const bool wg = h->p.mode == NCSB_MODE_PLAIN_WG;
    const bool spec = h->p.mode == NCSB_MODE_SPECTRAL;
    if (h->p.mode == NCSB_MODE_TC_TF32 || h->p.mode == NCSB_MODE_TC_BF16X3) {
        const bool bf = h->p.mode == NCSB_MODE_TC_BF16X3;
        e = cudaMemsetAsync(h->d_flag, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemsetAsync(flag)");
        a.flag = h->d_flag;
        const int per = h->p.ctas_per_sm > 0 ? h->p.ctas_per_sm
                                              : ncsb::tc_max_ctas_per_sm(bf, a.u0 != nullptr);
        const long long tpc = ncsb::tc_tiles_per_cta();
        long long grid = (long long)per * h->num_sms;
        if (grid > (a.n_tiles + tpc - 1) / tpc) grid = (a.n_tiles + tpc - 1) / tpc;
        if (grid < 1) grid = 1;
        e = ncsb::launch_tc(a, bf, (int)grid, s);
        if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
        return NCSB_OK;
    }
    int per_sm = h->p.ctas_per_sm > 0
                     ? h->p.ctas_per_sm
                     : (wg ? ncsb::plain_max_ctas_per_sm()
                           : (spec ? ncsb::spectral_max_ctas_per_sm(a.m, 0, a.u0 != nullptr,
                                                                   a.stacks != nullptr)
                                   : ncsb::warp_max_ctas_per_sm(a.m, 0)));
    // warp-per-tile CTAs hold 4 tiles at a time
    const long long tiles_per_cta = wg ? 1 : 4;
    long long grid = (long long)per_sm * h->num_sms;
    if (grid > (a.n_tiles + tiles_per_cta - 1) / tiles_per_cta)
        grid = (a.n_tiles + tiles_per_cta - 1) / tiles_per_cta;
    if (grid < 1) grid = 1;
    e = wg ? ncsb::launch_plain(a, (int)grid, s)
           : (spec ? ncsb::launch_spectral(a, (int)grid, h->p.ctas_per_sm, s)
                   : ncsb::launch_warp_blocks(a, (int)grid, h->p.ctas_per_sm, s));
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    return NCSB_OK;
}

}  // namespace

extern "C" {

void ncsb_default_params(ncsb_params* p) {
    if (!p) return;
    p->alpha = 0.2;
    p->max_iters = 200;
    p->m = 1;
    p->epsilon = 1e-5;
    p->c1 = 1e-4;
    p->min_step = 1e-6;
    p->mode = NCSB_MODE_SPECTRAL;
    p->ctas_per_sm = 0;
}

int ncsb_create(ncsb_handle** out, const ncsb_params* p) {
    if (!out) return NCSB_EINVAL;
    *out = nullptr;
    std::string why;
    int rc = check_params(p, &why);
    if (rc != NCSB_OK) return rc;
    ncsb_handle* h = new (std::nothrow) ncsb_handle();
    if (!h) return NCSB_EINVAL;
    h->p = *p;
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_msq, ncsb::kPix * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_queue, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_flag, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(h->d_flag, 0, sizeof(int32_t));
    if (e != cudaSuccess) {
        cudaFree(h->d_msq);
        cudaFree(h->d_queue);
        cudaFree(h->d_flag);
        delete h;
        return NCSB_ECUDA;
    }
    *out = h;
    return NCSB_OK;
}

int ncsb_set_params(ncsb_handle* h, const ncsb_params* p) {
    if (!h) return NCSB_EINVAL;
    std::string why;
    int rc = check_params(p, &why);
    if (rc != NCSB_OK) return fail(h, rc, why);
    h->p = *p;
    return NCSB_OK;
}

int ncsb_destroy(ncsb_handle* h) {
    if (!h) return NCSB_EINVAL;
    destroy_pipe(h->pipe);
    cudaFree(h->d_adu);
    cudaFree(h->d_msq);
    cudaFree(h->d_queue);
    cudaFree(h->d_flag);
    cudaFree(h->d_stacks);
    cudaFree(h->d_mk_lane);
    delete h;
    return NCSB_OK;
}

const char* ncsb_last_error(const ncsb_handle* h) { return h ? h->err.c_str() : "null handle"; }

int ncsb_set_otf_mask(ncsb_handle* h, const float* mask) {
    if (!h) return NCSB_EINVAL;
    if (!mask) return fail(h, NCSB_EINVAL, "mask is NULL");
    // natural order [kr][kc], scaled by 1/256; each kernel permutes it into
    // its own spectral layout when a CTA starts
    float tab[256];
    if (!build_msq(mask, tab)) return fail(h, NCSB_EINVAL, "mask has a non-finite value");
    cudaError_t e = cudaMemcpy(h->d_msq, tab, sizeof(tab), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemcpy(mask)");
    h->has_mask = true;
    return NCSB_OK;
}

int ncsb_num_tiles(int n_frames, int height, int width, int64_t* n_tiles) {
    if (!n_tiles) return NCSB_EINVAL;
    *n_tiles = 0;
    if (n_frames < 0) return NCSB_EINVAL;
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2) return NCSB_ESIZE;
    *n_tiles = (int64_t)n_frames * tiles_along(height) * tiles_along(width);
    return NCSB_OK;
}

int ncsb_reduce_noise(ncsb_handle* h, const float* images, int n_frames, int height, int width,
                      const float* gamma, int gamma_per_frame, float* out, int32_t* tile_iters,
                      int32_t* tile_status, double* tile_cost, int32_t* tile_evals,
                      void* stream) {
    if (!h) return NCSB_EINVAL;
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (n_frames < 0 || height <= 0 || width <= 0) return fail(h, NCSB_EINVAL, "bad shape");
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2)
        return fail(h, NCSB_ESIZE, "frames must be at least 14 x 14");
    if (n_frames == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!images || !gamma || !out) return fail(h, NCSB_EINVAL, "null buffer");
    ncsb::SolveArgs a{};
    a.tile_mode = 0;
    a.data = images;
    a.gamma = gamma;
    a.u0 = nullptr;
    a.gamma_frame_stride = gamma_per_frame ? (long long)height * width : 0;
    a.out = out;
    a.T = n_frames;
    a.H = height;
    a.W = width;
    a.tiles_x = tiles_along(height);
    a.tiles_y = tiles_along(width);
    a.n_tiles = (long long)n_frames * a.tiles_x * a.tiles_y;
    a.iters = tile_iters;
    a.status = tile_status;
    a.cost = tile_cost;
    a.evals = tile_evals;
    return launch(h, a, (cudaStream_t)stream);
}

}  // extern "C"

namespace {

// Create the pipeline's streams and events, and (re)size its buffers.
cudaError_t prepare_pipe(ncsb_handle* h, int n, size_t chunk_px, size_t gamma_px,
                         bool per_frame) {
    if (!h->pipe) {
        HostPipe* q = new (std::nothrow) HostPipe();
        if (!q) return cudaErrorMemoryAllocation;
        h->pipe = q;
        cudaError_t e = cudaMalloc(&q->d_queues, HostPipe::kMaxStreams * sizeof(unsigned long long));
        for (int k = 0; k < HostPipe::kMaxStreams && e == cudaSuccess; ++k) {
            e = cudaStreamCreateWithFlags(&q->st[k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q->done[k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q->start, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q->gamma_in, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            destroy_pipe(q);
            h->pipe = nullptr;
            return e;
        }
    }
    HostPipe* q = h->pipe;
    if (q->n != n || q->chunk_px < chunk_px || (per_frame && !q->per_frame)) {
        sync_pipe(q);  // a call that stopped on an error may have left work queued
        free_buffers(q);
        const size_t bytes = chunk_px * sizeof(float);
        for (int k = 0; k < n; ++k) {
            cudaError_t e = cudaMalloc(&q->d_in[k], bytes);
            if (e == cudaSuccess) e = cudaMalloc(&q->d_out[k], bytes);
            if (e == cudaSuccess && per_frame) e = cudaMalloc(&q->d_gf[k], bytes);
            if (e != cudaSuccess) {
                free_buffers(q);
                return e;
            }
        }
        q->n = n;
        q->chunk_px = chunk_px;
        q->per_frame = per_frame;
    }
    if (!per_frame && q->gamma_px < gamma_px) {
        sync_pipe(q);
        cudaFree(q->d_gamma);
        q->d_gamma = nullptr;
        q->gamma_px = 0;
        cudaError_t e = cudaMalloc(&q->d_gamma, gamma_px * sizeof(float));
        if (e != cudaSuccess) return e;
        q->gamma_px = gamma_px;
    }
    return cudaSuccess;
}

// The chunk loop of the host entries.  init(q, st0) queues work on stream 0
// that every chunk needs (a shared gamma map); stage(q, k, f0, n, st, a)
// queues chunk k's copy in (and conversion) on st and points a.data /
// a.gamma at the result.  Then each chunk is solved into d_out[k] and copied
// out on the same stream.  Returns after the last copy out; an error waits
// for the queued work before returning.
template <typename Init, typename Stage>
int run_host_pipe(ncsb_handle* h, int n_frames, int height, int width, bool per_frame,
                  float* out, int chunk_frames, int n_streams, cudaStream_t caller, Init init,
                  Stage stage) {
    const size_t frame_px = (size_t)height * width, fb = frame_px * sizeof(float);
    if (chunk_frames <= 0) {
        // about 40 chunks per stack (fastest on B200 for 200 x 512^2 and
        // close to it for 100 x 2048^2: short fill and drain, few per-chunk
        // gaps), at most 64 MB each
        const int cap = (int)(64.0e6 / (4.0 * (double)frame_px));
        chunk_frames = (n_frames + 20) / 40;
        if (chunk_frames > cap) chunk_frames = cap;
        if (chunk_frames < 1) chunk_frames = 1;
    }
    if (chunk_frames > n_frames) chunk_frames = n_frames;
    if (n_streams <= 0) n_streams = 4;
    if (n_streams > HostPipe::kMaxStreams) n_streams = HostPipe::kMaxStreams;
    cudaError_t e = prepare_pipe(h, n_streams, (size_t)chunk_frames * frame_px, frame_px,
                                 per_frame);
    if (e != cudaSuccess) return cuda_fail(h, e, "host pipeline set-up");
    HostPipe* q = h->pipe;
    // every stream starts after the caller's earlier work and after stream
    // 0's shared set-up
    e = cudaEventRecord(q->start, caller);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(q->st[0], q->start, 0);
    if (e == cudaSuccess) e = init(q, q->st[0]);
    if (e == cudaSuccess) e = cudaEventRecord(q->gamma_in, q->st[0]);
    for (int k = 1; k < n_streams && e == cudaSuccess; ++k)
        e = cudaStreamWaitEvent(q->st[k], q->gamma_in, 0);
    if (e != cudaSuccess) {
        sync_pipe(q);
        return cuda_fail(h, e, "host pipeline start");
    }
    for (int i = 0, f0 = 0; f0 < n_frames; ++i, f0 += chunk_frames) {
        const int n = n_frames - f0 < chunk_frames ? n_frames - f0 : chunk_frames;
        const int k = i % n_streams;
        cudaStream_t st = q->st[k];
        ncsb::SolveArgs a{};
        e = stage(q, k, f0, n, st, a);
        if (e != cudaSuccess) {
            sync_pipe(q);
            return cuda_fail(h, e, "host pipeline copy in");
        }
        a.tile_mode = 0;
        a.gamma_frame_stride = per_frame ? (long long)frame_px : 0;
        a.out = q->d_out[k];
        a.T = n;
        a.H = height;
        a.W = width;
        a.tiles_x = tiles_along(height);
        a.tiles_y = tiles_along(width);
        a.n_tiles = (long long)n * a.tiles_x * a.tiles_y;
        const int rc = launch(h, a, st, q->d_queues + k);
        if (rc != NCSB_OK) {
            sync_pipe(q);
            return rc;
        }
        e = cudaMemcpyAsync(out + (size_t)f0 * frame_px, q->d_out[k], (size_t)n * fb,
                            cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) {
            sync_pipe(q);
            return cuda_fail(h, e, "host pipeline copy out");
        }
    }
    // the caller's stream, and this call's return, wait for every stream
    for (int k = 0; k < n_streams && e == cudaSuccess; ++k) {
        e = cudaEventRecord(q->done[k], q->st[k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(caller, q->done[k], 0);
    }
    for (int k = 0; k < n_streams && e == cudaSuccess; ++k) e = cudaEventSynchronize(q->done[k]);
    if (e != cudaSuccess) {
        sync_pipe(q);
        return cuda_fail(h, e, "host pipeline finish");
    }
    return NCSB_OK;
}

}  // namespace

extern "C" {

int ncsb_reduce_noise_host(ncsb_handle* h, const float* images, int n_frames, int height,
                           int width, const float* gamma, int gamma_per_frame, float* out,
                           int chunk_frames, int n_streams, void* stream) {
    if (!h) return NCSB_EINVAL;
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (n_frames < 0 || height <= 0 || width <= 0) return fail(h, NCSB_EINVAL, "bad shape");
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2)
        return fail(h, NCSB_ESIZE, "frames must be at least 14 x 14");
    if (n_frames == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!images || !gamma || !out) return fail(h, NCSB_EINVAL, "null buffer");
    const size_t frame_px = (size_t)height * width, fb = frame_px * sizeof(float);
    const bool per_frame = gamma_per_frame != 0;
    // stream 0 copies a shared gamma map in before any chunk
    auto init = [&](HostPipe* q, cudaStream_t st0) {
        return per_frame ? cudaSuccess
                         : cudaMemcpyAsync(q->d_gamma, gamma, fb, cudaMemcpyHostToDevice, st0);
    };
    // chunk k: the photon frames (and per-frame gamma) straight into the solve's inputs
    auto stage = [&](HostPipe* q, int k, int f0, int n, cudaStream_t st, ncsb::SolveArgs& a) {
        cudaError_t e = cudaMemcpyAsync(q->d_in[k], images + (size_t)f0 * frame_px,
                                        (size_t)n * fb, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && per_frame)
            e = cudaMemcpyAsync(q->d_gf[k], gamma + (size_t)f0 * frame_px, (size_t)n * fb,
                                cudaMemcpyHostToDevice, st);
        a.data = q->d_in[k];
        a.gamma = per_frame ? q->d_gf[k] : q->d_gamma;
        return e;
    };
    return run_host_pipe(h, n_frames, height, width, per_frame, out, chunk_frames, n_streams,
                         (cudaStream_t)stream, init, stage);
}

int ncsb_reduce_noise_start(ncsb_handle* h, const float* images, int n_frames, int height,
                            int width, const float* gamma, int gamma_per_frame,
                            const float* u0_tiles, float* out, int32_t* tile_iters,
                            int32_t* tile_status, double* tile_cost, int32_t* tile_evals,
                            int32_t* tile_start, void* stream) {
    if (!h) return NCSB_EINVAL;
    if (h->p.mode != NCSB_MODE_SPECTRAL && h->p.mode != NCSB_MODE_TC_TF32 &&
        h->p.mode != NCSB_MODE_TC_BF16X3)
        return fail(h, NCSB_EINVAL, "a proposed start needs the spectral or a tensor-core form");
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (n_frames < 0 || height <= 0 || width <= 0) return fail(h, NCSB_EINVAL, "bad shape");
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2)
        return fail(h, NCSB_ESIZE, "frames must be at least 14 x 14");
    if (n_frames == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!images || !gamma || !out) return fail(h, NCSB_EINVAL, "null buffer");
    if (!u0_tiles) return fail(h, NCSB_EINVAL, "null proposal");
    ncsb::SolveArgs a{};
    a.tile_mode = 0;
    a.data = images;
    a.gamma = gamma;
    a.u0 = u0_tiles;
    a.start = tile_start;
    a.gamma_frame_stride = gamma_per_frame ? (long long)height * width : 0;
    a.out = out;
    a.T = n_frames;
    a.H = height;
    a.W = width;
    a.tiles_x = tiles_along(height);
    a.tiles_y = tiles_along(width);
    a.n_tiles = (long long)n_frames * a.tiles_x * a.tiles_y;
    a.iters = tile_iters;
    a.status = tile_status;
    a.cost = tile_cost;
    a.evals = tile_evals;
    return launch(h, a, (cudaStream_t)stream);
}

int ncsb_reduce_noise_adu(ncsb_handle* h, const float* adu, int n_frames, int height, int width,
                          const ncsb_calibration* cal, float* out, int32_t* tile_iters,
                          int32_t* tile_status, double* tile_cost, int32_t* tile_evals,
                          void* stream) {
    return ncsb_reduce_noise_adu_typed(h, adu, NCSB_ADU_F32, n_frames, height, width, cal, out,
                                       tile_iters, tile_status, tile_cost, tile_evals, stream);
}

int ncsb_reduce_noise_adu_typed(ncsb_handle* h, const void* adu, int adu_type, int n_frames,
                                int height, int width, const ncsb_calibration* cal, float* out,
                                int32_t* tile_iters, int32_t* tile_status, double* tile_cost,
                                int32_t* tile_evals, void* stream) {
    const int rc = check_adu_call(h, adu, adu_type, n_frames, height, width, cal, out);
    if (rc != NCSB_OK || n_frames == 0) return rc;
    // converted frames, then gamma (one map, or one per frame with several pairs)
    const size_t frame_px = (size_t)height * width, stack_px = (size_t)n_frames * frame_px;
    const bool multi = cal->n_levels > 1;
    const size_t need = stack_px + (multi ? stack_px : frame_px);
    cudaStream_t s = (cudaStream_t)stream;
    if (h->adu_px < need) {
        // earlier calls on the handle (on any stream) may still read the old buffer
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaFree(h->d_adu);
        h->d_adu = nullptr;
        h->adu_px = 0;
        if (e == cudaSuccess) e = cudaMalloc(&h->d_adu, need * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(h, e, "raw-ADU conversion buffer");
        h->adu_px = need;
    }
    float* d = h->d_adu;
    float* gam = h->d_adu + stack_px;
    cudaError_t e = ncsb::adu::launch_convert(adu, adu_type, n_frames, height, width, cal, d,
                                              multi ? gam : nullptr, multi ? nullptr : gam, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "raw-ADU conversion");
    ncsb::SolveArgs a{};
    a.tile_mode = 0;
    a.data = d;
    a.gamma = gam;
    a.gamma_frame_stride = multi ? (long long)frame_px : 0;
    a.out = out;
    a.T = n_frames;
    a.H = height;
    a.W = width;
    a.tiles_x = tiles_along(height);
    a.tiles_y = tiles_along(width);
    a.n_tiles = (long long)n_frames * a.tiles_x * a.tiles_y;
    a.iters = tile_iters;
    a.status = tile_status;
    a.cost = tile_cost;
    a.evals = tile_evals;
    return launch(h, a, s);
}

int ncsb_reduce_noise_adu_host(ncsb_handle* h, const void* adu, int adu_type, int n_frames,
                               int height, int width, const ncsb_calibration* cal, float* out,
                               int chunk_frames, int n_streams, void* stream) {
    const int rc = check_adu_call(h, adu, adu_type, n_frames, height, width, cal, out);
    if (rc != NCSB_OK || n_frames == 0) return rc;
    const size_t frame_px = (size_t)height * width;
    const size_t esize = adu_type == NCSB_ADU_F32 ? 4 : adu_type == NCSB_ADU_U16 ? 2 : 1;
    const bool multi = cal->n_levels > 1;
    const char* src = static_cast<const char*>(adu);
    // one pair: stream 0 computes the shared gamma map before any chunk
    auto init = [&](HostPipe* q, cudaStream_t st0) {
        return multi ? cudaSuccess
                     : ncsb::adu::launch_gamma_map(cal, (long long)frame_px, q->d_gamma, st0,
                                                   h->num_sms);
    };
    // chunk k: raw counts into d_out[k] (at most 4 bytes a pixel, so they fit;
    // the solve overwrites them only after the conversion, in stream order),
    // converted into d_in[k] (and per-frame gamma into d_gf[k])
    auto stage = [&](HostPipe* q, int k, int f0, int n, cudaStream_t st, ncsb::SolveArgs& a) {
        cudaError_t e = cudaMemcpyAsync(q->d_out[k], src + (size_t)f0 * frame_px * esize,
                                        (size_t)n * frame_px * esize, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = ncsb::adu::launch_convert(q->d_out[k], adu_type, n, height, width, cal, q->d_in[k],
                                          multi ? q->d_gf[k] : nullptr, nullptr, st);
        a.data = q->d_in[k];
        a.gamma = multi ? q->d_gf[k] : q->d_gamma;
        return e;
    };
    return run_host_pipe(h, n_frames, height, width, multi, out, chunk_frames, n_streams,
                         (cudaStream_t)stream, init, stage);
}

int ncsb_solve_tiles(ncsb_handle* h, const float* data_in, const float* gamma_in, const float* u0,
                     int64_t n_tiles, float* data_out, int32_t* iters, int32_t* status,
                     double* cost, int32_t* evals, void* stream) {
    if (!h) return NCSB_EINVAL;
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (n_tiles < 0) return fail(h, NCSB_EINVAL, "negative tile count");
    if (n_tiles == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!data_in || !gamma_in || !data_out) return fail(h, NCSB_EINVAL, "null buffer");
    ncsb::SolveArgs a{};
    a.tile_mode = 1;
    a.data = data_in;
    a.gamma = gamma_in;
    a.u0 = u0;
    a.out = data_out;
    a.n_tiles = n_tiles;
    a.iters = iters;
    a.status = status;
    a.cost = cost;
    a.evals = evals;
    return launch(h, a, (cudaStream_t)stream);
}

int ncsb_batch_set(ncsb_handle* h, const ncsb_stack* stacks, int n_stacks) {
    if (!h) return NCSB_EINVAL;
    if (!stacks || n_stacks < 1 || n_stacks > NCSB_MAX_STACKS)
        return fail(h, NCSB_EINVAL, "need 1..NCSB_MAX_STACKS stacks");
    std::vector<ncsb::StackDesc> desc(n_stacks);
    std::vector<float> mk((size_t)n_stacks * 256);
    std::vector<ncsb_optics> optics;  // stacks whose mask is built on the device
    std::vector<int> slots;
    long long total = 0;
    for (int i = 0; i < n_stacks; ++i) {
        const ncsb_stack& st = stacks[i];
        const std::string at = "stack " + std::to_string(i) + ": ";
        if (!st.images || !st.gamma || !st.out) return fail(h, NCSB_EINVAL, at + "null buffer");
        if (st.n_frames < 1 || st.height <= 0 || st.width <= 0)
            return fail(h, NCSB_EINVAL, at + "bad shape");
        if (st.height < NCSB_TILE - 2 || st.width < NCSB_TILE - 2)
            return fail(h, NCSB_ESIZE, at + "frames must be at least 14 x 14");
        if (!std::isfinite(st.alpha) || st.alpha < 0.0)
            return fail(h, NCSB_EINVAL, at + "alpha must be finite and >= 0");
        if (st.mask_from_optics) {
            if (!ncsb::masks::valid(st.optics)) return fail(h, NCSB_EINVAL, at + "bad optics");
            optics.push_back(st.optics);
            slots.push_back(i);
        } else {
            float nat[256];
            if (!build_msq(st.mask_shifted, nat))
                return fail(h, NCSB_EINVAL, at + "non-finite mask");
            lane_layout(nat, mk.data() + (size_t)i * 256);
        }
        ncsb::StackDesc& d = desc[i];
        d.data = st.images;
        d.gamma = st.gamma;
        d.out = st.out;
        d.gamma_frame_stride = st.gamma_per_frame ? (long long)st.height * st.width : 0;
        d.tile_begin = total;
        d.T = st.n_frames;
        d.H = st.height;
        d.W = st.width;
        d.tiles_x = tiles_along(st.height);
        d.tiles_y = tiles_along(st.width);
        d.alpha = (float)st.alpha;
        total += (long long)st.n_frames * d.tiles_x * d.tiles_y;
    }
    cudaError_t e = cudaSuccess;
    if (n_stacks > h->batch_cap) {
        cudaFree(h->d_stacks);
        cudaFree(h->d_mk_lane);
        h->d_stacks = nullptr;
        h->d_mk_lane = nullptr;
        h->batch_cap = 0;
        h->n_stacks = 0;
        e = cudaMalloc(&h->d_stacks, sizeof(ncsb::StackDesc) * n_stacks);
        if (e == cudaSuccess) e = cudaMalloc(&h->d_mk_lane, sizeof(float) * 256 * n_stacks);
        if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc(batch)");
        h->batch_cap = n_stacks;
    }
    e = cudaMemcpy(h->d_stacks, desc.data(), sizeof(ncsb::StackDesc) * n_stacks,
                   cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(h->d_mk_lane, mk.data(), sizeof(float) * mk.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemcpy(batch)");
    if (!optics.empty()) {
        // overwrite those stacks' tables with masks built on the device
        const int no = (int)optics.size();
        ncsb_optics* d_optics = nullptr;
        int* d_slots = nullptr;
        e = cudaMalloc(&d_optics, sizeof(ncsb_optics) * no);
        if (e == cudaSuccess) e = cudaMalloc(&d_slots, sizeof(int) * no);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_optics, optics.data(), sizeof(ncsb_optics) * no,
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_slots, slots.data(), sizeof(int) * no, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = ncsb::masks::launch_masks(d_optics, no, nullptr, h->d_mk_lane, d_slots, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(d_optics);
        cudaFree(d_slots);
        if (e != cudaSuccess) return cuda_fail(h, e, "device masks");
    }
    h->n_stacks = n_stacks;
    h->batch_tiles = total;
    // resolve the kernel variants' attributes now, outside any stream capture
    ncsb::spectral_max_ctas_per_sm(h->p.m, 0, false, true);
    ncsb::spectral_max_ctas_per_sm(h->p.m, 0, true, true);
    return NCSB_OK;
}

int ncsb_batch_num_tiles(const ncsb_handle* h, int64_t* n_tiles) {
    if (!h || !n_tiles) return NCSB_EINVAL;
    *n_tiles = h->batch_tiles;
    return NCSB_OK;
}

int ncsb_batch_reduce_noise(ncsb_handle* h, const float* u0_tiles, int32_t* tile_iters,
                            int32_t* tile_status, double* tile_cost, int32_t* tile_evals,
                            int32_t* tile_start, void* stream) {
    if (!h) return NCSB_EINVAL;
    if (h->p.mode != NCSB_MODE_SPECTRAL && h->p.mode != NCSB_MODE_TC_TF32 &&
        h->p.mode != NCSB_MODE_TC_BF16X3)
        return fail(h, NCSB_EINVAL, "batched launches need the spectral or a tensor-core form");
    if (h->n_stacks < 1) return fail(h, NCSB_EINVAL, "call ncsb_batch_set first");
    ncsb::SolveArgs a{};
    a.tile_mode = 0;
    a.stacks = h->d_stacks;
    a.n_stacks = h->n_stacks;
    a.mk_lane = h->d_mk_lane;
    a.u0 = u0_tiles;
    a.start = tile_start;
    a.n_tiles = h->batch_tiles;
    a.iters = tile_iters;
    a.status = tile_status;
    a.cost = tile_cost;
    a.evals = tile_evals;
    return launch(h, a, (cudaStream_t)stream);
}

int ncsb_net_infer_batch(const float* params, const ncsb_handle* h, float* u0_tiles,
                         void* stream) {
    if (!params || !h || !u0_tiles) return NCSB_EINVAL;
    if (h->n_stacks < 1) return NCSB_EINVAL;
    return ncsb::net::launch_infer_batch(params, h->d_stacks, h->n_stacks, h->batch_tiles,
                                         u0_tiles, (cudaStream_t)stream);
}

int ncsb_net_infer_batch_tc(const float* params, const ncsb_handle* h, float* u0_tiles,
                            int32_t* status, void* stream) {
    if (!params || !h || !u0_tiles) return NCSB_EINVAL;
    if (h->n_stacks < 1) return NCSB_EINVAL;
    return ncsb::nettc::launch_batch(params, h->d_stacks, h->n_stacks, h->batch_tiles, u0_tiles,
                                     status, false, (cudaStream_t)stream);
}

int ncsb_net_infer_batch_tc_fp8(const float* params, const ncsb_handle* h, float* u0_tiles,
                                int32_t* status, void* stream) {
    if (!params || !h || !u0_tiles) return NCSB_EINVAL;
    if (h->n_stacks < 1) return NCSB_EINVAL;
    return ncsb::nettc::launch_batch(params, h->d_stacks, h->n_stacks, h->batch_tiles, u0_tiles,
                                     status, true, (cudaStream_t)stream);
}

}  // extern "C"
