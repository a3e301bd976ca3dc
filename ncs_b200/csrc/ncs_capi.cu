// ncs_capi.cu -- the extern "C" ABI of libncs_b200.so (declared in
// include/ncs_b200.h).  Owns the handle: solver parameters, the device mask
// table and the work-queue counter; mirrors ncsSRInitialize / ncsSRCleanup
// (clib/pyCNCS/ncs.c:394-446, :307-327) for the device.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/ncs_b200.h"
#include "ncs_internal.cuh"

namespace ncsb {
cudaError_t launch_plain(const SolveArgs& args, int grid, cudaStream_t stream);
int plain_max_ctas_per_sm();
cudaError_t launch_warp_blocks(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int warp_max_ctas_per_sm(int m, int blocks);
cudaError_t launch_spectral(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int spectral_max_ctas_per_sm(int m, int blocks);
}  // namespace ncsb

struct ncsb_handle {
    ncsb_params p;
    int device = 0;
    int num_sms = 1;
    bool has_mask = false;
    float* d_msq = nullptr;                 // [256] M^2/256, kernel spectral layout
    unsigned long long* d_queue = nullptr;  // work counter
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

int check_params(const ncsb_params* p, std::string* why) {
    if (!p) { *why = "params is NULL"; return NCSB_EINVAL; }
    if (!std::isfinite(p->alpha) || p->alpha < 0.0) { *why = "alpha must be finite and >= 0"; return NCSB_EINVAL; }
    if (p->max_iters < 0) { *why = "max_iters must be >= 0"; return NCSB_EINVAL; }
    if (p->m < 1 || p->m > ncsb::kMaxM) { *why = "m must be in 1..8"; return NCSB_EINVAL; }
    if (!(p->epsilon >= 0.0)) { *why = "epsilon must be >= 0"; return NCSB_EINVAL; }
    if (!(p->c1 > 0.0 && p->c1 < 1.0)) { *why = "c1 must be in (0, 1)"; return NCSB_EINVAL; }
    if (!(p->min_step > 0.0)) { *why = "min_step must be > 0"; return NCSB_EINVAL; }
    if (p->mode != NCSB_MODE_PLAIN && p->mode != NCSB_MODE_PLAIN_WG && p->mode != NCSB_MODE_SPECTRAL) { *why = "unsupported mode"; return NCSB_EINVAL; }
    if (p->ctas_per_sm < 0) { *why = "ctas_per_sm must be >= 0"; return NCSB_EINVAL; }
    return NCSB_OK;
}

int tiles_along(int n) {
    // len(range(0, n + 2, 14)) with the last origin clamped to n + 2 - 16
    // and the walk stopped after it (ncs.c:71-86, :136-142).
    const int last = n + 2 - NCSB_TILE;
    int count = 0;
    for (int b = 0;; b += 14) {
        ++count;
        if (b >= last) break;
    }
    return count;
}

int launch(ncsb_handle* h, ncsb::SolveArgs& a, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(h->d_queue, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemsetAsync(queue)");
    a.queue = h->d_queue;
    a.msq = h->d_msq;
    a.alpha = (float)h->p.alpha;
    a.eps = (float)h->p.epsilon;
    a.c1 = (float)h->p.c1;
    a.min_step = (float)h->p.min_step;
    a.max_iters = h->p.max_iters;
    a.m = h->p.m;
    const bool wg = h->p.mode == NCSB_MODE_PLAIN_WG;
    const bool spec = h->p.mode == NCSB_MODE_SPECTRAL;
    int per_sm = h->p.ctas_per_sm > 0
                     ? h->p.ctas_per_sm
                     : (wg ? ncsb::plain_max_ctas_per_sm()
                           : (spec ? ncsb::spectral_max_ctas_per_sm(a.m, 0)
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
    p->m = 2;
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
    if (e != cudaSuccess) {
        cudaFree(h->d_msq);
        cudaFree(h->d_queue);
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
    cudaFree(h->d_msq);
    cudaFree(h->d_queue);
    delete h;
    return NCSB_OK;
}

const char* ncsb_last_error(const ncsb_handle* h) { return h ? h->err.c_str() : "null handle"; }

int ncsb_set_otf_mask(ncsb_handle* h, const float* mask) {
    if (!h) return NCSB_EINVAL;
    if (!mask) return fail(h, NCSB_EINVAL, "mask is NULL");
    // M^2, symmetrised over k -> -k: for real u the noise term only sees the
    // symmetric part (|U_k| = |U_-k|), and the kernel's real-output inverse
    // transform relies on it.  A mask passing checkOTFMask is unchanged.
    double m2[16][16];
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 16; ++j) {
            const double a = mask[i * 16 + j], b = mask[((16 - i) & 15) * 16 + ((16 - j) & 15)];
            if (!std::isfinite(a)) return fail(h, NCSB_EINVAL, "mask has a non-finite value");
            m2[i][j] = 0.5 * (a * a + b * b);
        }
    // Natural order [kr][kc], scaled by 1/256; each kernel permutes it into
    // its own spectral layout when a CTA starts.
    float tab[256];
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 16; ++j) tab[i * 16 + j] = (float)(m2[i][j] / 256.0);
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
    if (!images || !gamma || !out) return fail(h, NCSB_EINVAL, "null buffer");
    if (n_frames < 0 || height <= 0 || width <= 0) return fail(h, NCSB_EINVAL, "bad shape");
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2)
        return fail(h, NCSB_ESIZE, "frames must be at least 14 x 14");
    if (n_frames == 0) return NCSB_OK;
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

int ncsb_solve_tiles(ncsb_handle* h, const float* data_in, const float* gamma_in, const float* u0,
                     int64_t n_tiles, float* data_out, int32_t* iters, int32_t* status,
                     double* cost, int32_t* evals, void* stream) {
    if (!h) return NCSB_EINVAL;
    if (!h->has_mask) return fail(h, NCSB_ENOMASK, "call ncsb_set_otf_mask first");
    if (!data_in || !gamma_in || !data_out) return fail(h, NCSB_EINVAL, "null buffer");
    if (n_tiles < 0) return fail(h, NCSB_EINVAL, "negative tile count");
    if (n_tiles == 0) return NCSB_OK;
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

}  // extern "C"
