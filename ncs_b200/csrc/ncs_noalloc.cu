// ncs_noalloc.cu -- ncsb_reduce_noise_noalloc: the whole-stack solve without a
// handle and without any device allocation.
//
// Who needs it: code that must not call cudaMalloc once it is running, e.g.
// a plug-in inside a microscope acquisition or image-server process whose
// host application owns the whole GPU memory budget (through its own pool
// allocator), or a real-time pipeline that has a "no device allocation after
// start-up" rule because cudaMalloc can synchronise the device and stall the
// camera stream.  Such callers cannot create an ncsb_handle (ncsb_create
// allocates the work counter and the mask table), so this entry point keeps
// that scratch in a fixed file-scope __device__ array instead.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; each call re-initialises the work counter and the mask
// table on its own stream before the launch, with a one-block kernel that
// receives the table by value (no host-to-device copy, so the host never
// waits for the stream).  Calls that overlap on the GPU (two streams, or two
// host threads) race on it.  The device address of the array is looked up
// once per device and kept for the life of the process, so the entry must
// not be used across cudaDeviceReset on that device.
#include <cmath>
#include <mutex>

#include "../../include/ncs_b200.h"
#include "ncs_internal.cuh"

namespace ncsb {
cudaError_t launch_plain(const SolveArgs& args, int grid, cudaStream_t stream);
int plain_max_ctas_per_sm();
cudaError_t launch_warp_blocks(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int warp_max_ctas_per_sm(int m, int blocks);
cudaError_t launch_spectral(const SolveArgs& args, int grid, int blocks, cudaStream_t stream);
int spectral_max_ctas_per_sm(int m, int blocks, bool warm, bool batch);
}  // namespace ncsb

using ncsb::tiles_along;

namespace {

// Layout of the static scratch: [0, 8) work counter, [256, 1280) the
// 256-entry M^2/256 table in natural [kr][kc] order (the table
// ncsb_set_otf_mask builds; each kernel remaps it to its own layout).  Capacity is
// NCSB_NOALLOC_SCRATCH_BYTES (4 KiB); every GPU that loads the library holds
// it until the process exits.
constexpr size_t kQueueOffset = 0;
constexpr size_t kTableOffset = 256;
constexpr size_t kTableBytes = ncsb::kPix * sizeof(float);
static_assert(NCSB_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch capacity");

static __device__ __align__(256) unsigned char g_scratch[NCSB_NOALLOC_SCRATCH_BYTES];

struct DeviceSetup {
    bool done = false;
    unsigned char* scratch = nullptr;  // device address of g_scratch on this device
    int num_sms = 0;
    int ctas_per_sm = 0;
};

// The M^2/256 table travels as a kernel argument (1 KiB, by value).
struct TableArg {
    float v[ncsb::kPix];
};

// Writes the mask table into the scratch array and resets the work counter.
__global__ void noalloc_init_kernel(TableArg table, unsigned char* scratch) {
    float* dst = reinterpret_cast<float*>(scratch + kTableOffset);
    for (int i = threadIdx.x; i < ncsb::kPix; i += blockDim.x) dst[i] = table.v[i];
    if (threadIdx.x == 0) *reinterpret_cast<unsigned long long*>(scratch + kQueueOffset) = 0ull;
}

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// Once per device, with that device current: resolve the device address of
// the scratch array (its name in host code is only a host-side stand-in) and
// cache the launch geometry.
int setup_current_device(DeviceSetup** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return NCSB_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return NCSB_EINVAL;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& s = g_setup[dev];
    if (!s.done) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || ptr == nullptr)
            return NCSB_ECUDA;
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return NCSB_ECUDA;
        s.scratch = static_cast<unsigned char*>(ptr);
        s.num_sms = sms > 0 ? sms : 1;
        s.ctas_per_sm = ncsb::plain_max_ctas_per_sm();
        s.done = true;
    }
    *out = &s;
    return NCSB_OK;
}

bool params_ok(const ncsb_params* p) {
    return p && std::isfinite(p->alpha) && p->alpha >= 0.0 && p->max_iters >= 0 && p->m >= 1 &&
           p->m <= ncsb::kMaxM && p->epsilon >= 0.0 && p->c1 > 0.0 && p->c1 < 1.0 &&
           p->min_step > 0.0 &&
           (p->mode == NCSB_MODE_PLAIN || p->mode == NCSB_MODE_PLAIN_WG ||
            p->mode == NCSB_MODE_SPECTRAL) &&
           p->ctas_per_sm >= 0;
}

}  // namespace

extern "C" int ncsb_reduce_noise_noalloc(const ncsb_params* p, const float* mask_shifted_host,
                                         const float* images, int n_frames, int height,
                                         int width, const float* gamma, int gamma_per_frame,
                                         float* out, int32_t* tile_iters, int32_t* tile_status,
                                         double* tile_cost, int32_t* tile_evals, void* stream) {
    if (!params_ok(p) || !mask_shifted_host) return NCSB_EINVAL;
    if (n_frames < 0 || height <= 0 || width <= 0) return NCSB_EINVAL;
    if (height < NCSB_TILE - 2 || width < NCSB_TILE - 2) return NCSB_ESIZE;
    // Everything this call keeps on the device must fit the static array.
    if (kTableOffset + kTableBytes > (size_t)NCSB_NOALLOC_SCRATCH_BYTES) return NCSB_ESCRATCH;
    if (n_frames == 0) return NCSB_OK;  // nothing read or written: buffers may be null
    if (!images || !gamma || !out) return NCSB_EINVAL;

    DeviceSetup* dev = nullptr;
    int rc = setup_current_device(&dev);
    if (rc != NCSB_OK) return rc;

    // M^2 symmetrised over k -> -k and scaled by 1/256, natural order (the
    // table ncsb_set_otf_mask builds).
    TableArg table;
    for (int kr = 0; kr < 16; ++kr) {
        for (int kc = 0; kc < 16; ++kc) {
            const double a = mask_shifted_host[kr * 16 + kc];
            const double b = mask_shifted_host[((16 - kr) & 15) * 16 + ((16 - kc) & 15)];
            if (!std::isfinite(a) || !std::isfinite(b)) return NCSB_EINVAL;
            table.v[kr * 16 + kc] = (float)(0.5 * (a * a + b * b) / 256.0);
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* scratch = dev->scratch;
    noalloc_init_kernel<<<1, 256, 0, s>>>(table, scratch);
    if (cudaGetLastError() != cudaSuccess) return NCSB_ECUDA;

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
    a.queue = reinterpret_cast<unsigned long long*>(scratch + kQueueOffset);
    a.msq = reinterpret_cast<const float*>(scratch + kTableOffset);
    a.alpha = (float)p->alpha;
    a.eps = (float)p->epsilon;
    a.c1 = (float)p->c1;
    a.min_step = (float)p->min_step;
    a.max_iters = p->max_iters;
    a.m = p->m;
    const bool wg = p->mode == NCSB_MODE_PLAIN_WG;
    const bool spec = p->mode == NCSB_MODE_SPECTRAL;
    const int per_sm = p->ctas_per_sm > 0
                           ? p->ctas_per_sm
                           : (wg ? dev->ctas_per_sm
                                 : (spec ? ncsb::spectral_max_ctas_per_sm(a.m, 0, false, false)
                                         : ncsb::warp_max_ctas_per_sm(a.m, 0)));
    const long long tiles_per_cta = wg ? 1 : 4;
    long long grid = (long long)per_sm * dev->num_sms;
    if (grid > (a.n_tiles + tiles_per_cta - 1) / tiles_per_cta)
        grid = (a.n_tiles + tiles_per_cta - 1) / tiles_per_cta;
    if (grid < 1) grid = 1;
    const cudaError_t e = wg     ? ncsb::launch_plain(a, (int)grid, s)
                          : spec ? ncsb::launch_spectral(a, (int)grid, p->ctas_per_sm, s)
                                 : ncsb::launch_warp_blocks(a, (int)grid, p->ctas_per_sm, s);
    return e == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}
