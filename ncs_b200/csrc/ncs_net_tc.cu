// ncs_net_tc.cu -- warm-start network inference on the 5th-generation tensor
// cores (tcgen05, sm_100a): the same network as ncs_net.cu's FP32 inference,
// as implicit GEMMs with BF16 operands and FP32 accumulators in tensor memory.
//
// Per 16x16 tile, positions live on the zero-bordered 18 x 18 plane
// (row-major, index P).  The outputs of a 3x3 layer at the 288 positions
// P = 18..305 (plane rows 1..16, all 18 columns; the two border columns are
// computed and discarded) are, for each tap (ky, kx), a GEMM
//     D[q][co] += sum_ci A[q + 18 + (ky-1)*18 + (kx-1)][ci] * W[tap][ci][co]
// so the tap is a shift of the A operand's start position: one shared-memory
// matrix descriptor per tap over the same activation buffer.  M = 128
// (3 blocks cover the 288 positions), N = 32 (N = 16 for the 1-channel last
// layer, weights zero-padded), K = 16 per instruction, 2 per 32 channels.
// The first layer (2 input channels) is one GEMM with an im2col operand,
// K = 18 taps x channels padded to 32.
//
// Shared-memory operands are K-major without swizzle: 8 consecutive
// positions x 8 channels (16 B each) form a core matrix, so an activation
// buffer is [channel chunk][position][8] BF16 with the leading byte offset
// (between K halves) = the chunk stride and the stride byte offset (between
// 8-row groups) = 128 B.  The epilogue reads each accumulator row from tensor
// memory (thread t of the 128 owns row t of every M block), adds the bias,
// applies ReLU, rounds to BF16 and writes the next layer's operand -- zeros at
// the plane's border positions, which are the next layer's zero padding.
//
// A layer's MMAs have finished reading their input before its epilogue
// runs, so the epilogue overwrites that input in place: one activation
// buffer per tile.  A CTA (4 warps) keeps two tiles in flight in two slots,
// each with its buffer, 128 tensor-memory columns and an mbarrier, and
// alternates between them: wait for a slot's MMAs, run its epilogue, issue
// its next layer (or start its next tile), turn to the other slot -- so one
// slot's epilogue runs while the other slot's MMAs do.  Two such CTAs share
// an SM, persistent over tiles.  Thread 0 issues the MMAs and commits them
// to the slot's mbarrier, which all threads wait on.  Every wait is bounded;
// a timed-out wait sets the caller's status flag, drains the outstanding
// MMAs with bounded waits, frees the tensor memory and ends the kernel.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ncs_b200.h"
#include "ncs_internal.cuh"

namespace ncsb {
namespace nettc {

constexpr int kC = 32;
constexpr int kThreads = 128;
constexpr int kPlane = 18;
constexpr int kQ = 384;                  // 3 M blocks of 128 output positions
constexpr int kPos = 424;                // activation positions incl. shift margins
constexpr int kChunkA = kPos * 16;       // bytes per 8-channel chunk of an activation buffer
constexpr int kActBytes = 4 * kChunkA;   // 32 channels
constexpr int kW1Bytes = 4 * 32 * 16;            // layer 1: K 32 x N 32
constexpr int kWtapBytes = 4 * 32 * 16;          // layers 2, 3: per tap K 32 x N 32
constexpr int kW4tapBytes = 4 * 16 * 16;         // layer 4: per tap K 32 x N 16
constexpr float kStartFrac = 0.05f;
constexpr int kSlots = 2;                // tiles in flight per CTA
constexpr unsigned kTmemCols = 256;      // 128 columns per slot
constexpr long long kWaitTries = 1ll << 22;  // mbarrier polls before giving up (seconds)

// shared-memory plan (bytes, all 128-B aligned)
constexpr int kOffW1 = 0;
constexpr int kOffW2 = kOffW1 + kW1Bytes;
constexpr int kOffW3 = kOffW2 + 9 * kWtapBytes;
constexpr int kOffW4 = kOffW3 + 9 * kWtapBytes;
constexpr int kOffAct = kOffW4 + 9 * kW4tapBytes;             // one buffer per slot
// the layer-1 im2col operand lives in the slot's activation buffer at
// positions 19..402 -- the range every epilogue rewrites -- so the zero
// border positions of the buffer are never touched
constexpr int kIm2colPos = 19;
constexpr int kOffBias = kOffAct + kSlots * kActBytes;        // 3 x 32 + 1 floats
constexpr int kOffTile = kOffBias + 128 * 4;                  // per slot d, gamma, x0, x1
constexpr int kTileBytes = 4 * 256 * 4;
constexpr int kSmemBytes = kOffTile + kSlots * kTileBytes;

struct Src {
    int tile_mode;
    const float* d;
    const float* gamma;
    long long gamma_frame_stride;
    int H, W, tiles_x, tiles_y;
    long long n_tiles;
    const StackDesc* stacks;  // batched stacks (stack mode), else null
    int n_stacks;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no swizzle (layout type 0), Blackwell descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id,
                                    uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool wait_bounded(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitTries; ++i)
        if (try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Store 32 channels of one position into a [chunk][pos][8] BF16 buffer.
__device__ __forceinline__ void store_pos(unsigned char* buf, int chunk_bytes, int pos,
                                          const float (&v)[32]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint4 w;
        w.x = pack2(v[8 * k + 0], v[8 * k + 1]);
        w.y = pack2(v[8 * k + 2], v[8 * k + 3]);
        w.z = pack2(v[8 * k + 4], v[8 * k + 5]);
        w.w = pack2(v[8 * k + 6], v[8 * k + 7]);
        *reinterpret_cast<uint4*>(buf + k * chunk_bytes + pos * 16) = w;
    }
}

// The 54 MMAs of a 3x3 layer over one slot: 3 M blocks x 9 taps x 2 K steps,
// every operand offset and accumulate flag a compile-time constant (the
// issuing thread is on the critical path: the other threads wait at the next
// barrier while it issues).  NOut = 32, or 16 for the last layer.
template <int NOut>
__device__ __forceinline__ void issue_taps(uint32_t td, uint64_t a0, uint64_t b0) {
    constexpr uint32_t id = idesc(128, NOut);
    constexpr int tap_bytes = NOut == 32 ? kWtapBytes : kW4tapBytes;
    constexpr int wchunk = NOut * 16;
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int tap = 0; tap < 9; ++tap)
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const int pos = kPlane + 128 * m + (tap / 3 - 1) * kPlane + (tap % 3 - 1) + 1;
                mma(td + m * NOut, a0 + (((2 * ks) * kChunkA + pos * 16) >> 4),
                    b0 + ((tap * tap_bytes + (2 * ks) * wchunk) >> 4), id, (tap | ks) != 0);
            }
}

__global__ void __launch_bounds__(kThreads, 2)
    infer_tc(const Src src, const float* __restrict__ params, float* __restrict__ u0,
             int32_t* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar[kSlots];
    __shared__ uint32_t tmem_base_s;
    __shared__ float red[8];
    const int t = threadIdx.x, warp = t >> 5;

    // ---- weights -> BF16 operand layouts, biases, zeroed activations --------
    const float* w1 = params;
    const float* b1 = w1 + 2 * 9 * kC;
    const float* w2 = b1 + kC;
    const float* b2 = w2 + kC * 9 * kC;
    const float* w3 = b2 + kC;
    const float* b3 = w3 + kC * 9 * kC;
    const float* w4 = b3 + kC;
    const float* b4 = w4 + kC * 9;
    __nv_bfloat16* sW1 = reinterpret_cast<__nv_bfloat16*>(sm + kOffW1);
    // layer 1, B[k][co] with k = tap * 2 + ci (18 used of 32): [k chunk][co][8]
    for (int i = t; i < 32 * 32; i += kThreads) {
        const int k = i >> 5, co = i & 31;
        const float v = k < 18 ? w1[((k & 1) * 9 + (k >> 1)) * kC + co] : 0.0f;
        sW1[(k >> 3) * 256 + co * 8 + (k & 7)] = __float2bfloat16_rn(v);
    }
    for (int l = 0; l < 2; ++l) {
        const float* w = l == 0 ? w2 : w3;
        __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(sm + (l == 0 ? kOffW2 : kOffW3));
        for (int i = t; i < 9 * 32 * 32; i += kThreads) {
            const int tap = i / 1024, rem = i - tap * 1024, ci = rem >> 5, co = rem & 31;
            sW[tap * 1024 + (ci >> 3) * 256 + co * 8 + (ci & 7)] =
                __float2bfloat16_rn(w[(ci * 9 + tap) * kC + co]);
        }
    }
    {
        __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(sm + kOffW4);
        for (int i = t; i < 9 * 32 * 16; i += kThreads) {
            const int tap = i / 512, rem = i - tap * 512, ci = rem >> 4, co = rem & 15;
            sW[tap * 512 + (ci >> 3) * 128 + co * 8 + (ci & 7)] =
                __float2bfloat16_rn(co == 0 ? w4[ci * 9 + tap] : 0.0f);
        }
    }
    float* sBias = reinterpret_cast<float*>(sm + kOffBias);
    for (int i = t; i < 97; i += kThreads)
        sBias[i] = i < 32 ? b1[i] : (i < 64 ? b2[i - 32] : (i < 96 ? b3[i - 64] : b4[0]));
    for (int i = t; i < kSlots * kActBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(sm + kOffAct)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (t == 0) {
        for (int sl = 0; sl < kSlots; ++sl)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[sl]))
                         : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_s)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base_s;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;  // this warp's TMEM lanes
    const uint32_t sW1a = smem_u32(sm + kOffW1), sW2a = smem_u32(sm + kOffW2);
    const uint32_t sW3a = smem_u32(sm + kOffW3), sW4a = smem_u32(sm + kOffW4);
    const long long per_frame = (long long)src.tiles_x * src.tiles_y;
    const long long stride = (long long)kSlots * gridDim.x;  // tiles between a slot's tiles

    // per-slot state, block-uniform: current tile, next layer to wait for,
    // mbarrier phase, feature scale; and this thread's prefetched pixels
    long long tile_s[kSlots] = {};
    int layer_s[kSlots] = {};
    uint32_t phase_s[kSlots] = {};
    float scale_s[kSlots] = {};
    float dv[kSlots][2] = {}, gv[kSlots][2] = {};
    bool alive = true;

    // this thread's two pixels of a tile (the solvers' segmentation)
    auto gather = [&](long long tile, float (&dvo)[2], float (&gvo)[2]) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int p = t + 128 * h, r = p >> 4, c = p & 15;
            if (src.tile_mode) {
                dvo[h] = src.d[tile * 256 + p];
                gvo[h] = src.gamma[tile * 256 + p];
            } else {
                const float* sd = src.d;
                const float* sgam = src.gamma;
                long long gstride = src.gamma_frame_stride, lt = tile, pf = per_frame;
                int H = src.H, W = src.W, ty = src.tiles_y;
                if (src.stacks) {  // batched: the last stack whose first tile is <= tile
                    int lo = 0, hi = src.n_stacks - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (src.stacks[mid].tile_begin <= tile) lo = mid;
                        else hi = mid - 1;
                    }
                    const StackDesc& st = src.stacks[lo];
                    sd = st.data;
                    sgam = st.gamma;
                    gstride = st.gamma_frame_stride;
                    lt = tile - st.tile_begin;
                    H = st.H;
                    W = st.W;
                    ty = st.tiles_y;
                    pf = (long long)st.tiles_x * st.tiles_y;
                }
                const int f = (int)(lt / pf);
                const int rem = (int)(lt - (long long)f * pf);
                const int ti = rem / ty, tj = rem - ti * ty;
                const int yy = clampi(tile_origin(ti, H) + r - 1, 0, H - 1);
                const int xx = clampi(tile_origin(tj, W) + c - 1, 0, W - 1);
                dvo[h] = sd[(long long)f * H * W + (long long)yy * W + xx];
                gvo[h] = sgam[(long long)f * gstride + (long long)yy * W + xx];
            }
        }
    };

    // features of slot sl's tile from the gathered pixels, and the layer-1
    // im2col operand in the slot's activation buffer (whose previous reader,
    // the slot's last layer, has completed)
    auto build = [&](int sl) {
        float* sD = reinterpret_cast<float*>(sm + kOffTile + sl * kTileBytes);
        float* sG = sD + 256;
        float* sX0 = sG + 256;
        float* sX1 = sX0 + 256;
        float s1 = dv[sl][0] + dv[sl][1], s2 = dv[sl][0] * dv[sl][0] + dv[sl][1] * dv[sl][1];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        __syncthreads();  // earlier readers of red and of this slot's tile data are done
        if ((t & 31) == 0) {
            red[warp] = s1;
            red[4 + warp] = s2;
        }
        __syncthreads();
        const float mu = (red[0] + red[1] + red[2] + red[3]) * (1.0f / 256.0f);
        const float sd = sqrtf(fmaxf((red[4] + red[5] + red[6] + red[7]) * (1.0f / 256.0f) -
                                     mu * mu, 0.0f)) + 1.0f;
        scale_s[sl] = sd;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int p = t + 128 * h;
            sD[p] = dv[sl][h];
            sG[p] = gv[sl][h];
            sX0[p] = (dv[sl][h] - mu) / sd;
            sX1[p] = sqrtf(fmaxf(dv[sl][h], 0.0f) + fmaxf(gv[sl][h], 0.0f)) / sd;
        }
        __syncthreads();
        unsigned char* im2col = sm + kOffAct + sl * kActBytes + kIm2colPos * 16;
#pragma unroll 1
        for (int m = 0; m < 3; ++m) {
            const int q = 128 * m + t, P = q + kPlane;
            const int R = P / kPlane, Cc = P - R * kPlane;
            float v[32];
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                const int rr = R + tap / 3 - 1, cc = Cc + tap % 3 - 1;
                const bool in = rr >= 1 && rr <= 16 && cc >= 1 && cc <= 16;
                const int px = in ? (rr - 1) * 16 + (cc - 1) : 0;
                v[2 * tap] = in ? sX0[px] : 0.0f;
                v[2 * tap + 1] = in ? sX1[px] : 0.0f;
            }
#pragma unroll
            for (int k = 18; k < 32; ++k) v[k] = 0.0f;
            store_pos(im2col, kChunkA, q, v);
        }
    };

    // make the slot's operand writes visible to the tensor core, then thread
    // 0 issues the layer's MMAs and commits them to the slot's mbarrier
    auto issue = [&](int sl, int layer) {
        fence_async_smem();
        fence_before();
        __syncthreads();
        if (t == 0) {
            // descriptors are built once per layer; an operand offset is added
            // to the start-address field (shared addresses < 256 KB, so the
            // 14-bit field never carries)
            fence_after();
            const uint32_t act_a = smem_u32(sm + kOffAct + sl * kActBytes);
            const uint32_t td = tmem + (uint32_t)(sl * 128);
            if (layer == 0) {
                constexpr uint32_t id = idesc(128, 32);
                const uint64_t a0 = sdesc(act_a + kIm2colPos * 16, kChunkA, 128);
                const uint64_t b0 = sdesc(sW1a, 512, 128);
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int ks = 0; ks < 2; ++ks)
                        mma(td + m * 32, a0 + (((2 * ks) * kChunkA + 128 * m * 16) >> 4),
                            b0 + (((2 * ks) * 512) >> 4), id, ks);
            } else if (layer < 3) {
                issue_taps<32>(td, sdesc(act_a, kChunkA, 128),
                               sdesc(layer == 1 ? sW2a : sW3a, 512, 128));
            } else {
                issue_taps<16>(td, sdesc(act_a, kChunkA, 128), sdesc(sW4a, 256, 128));
            }
            commit(smem_u32(&bar[sl]));
        }
    };

    // all threads: wait for the slot's committed MMAs (block-uniform outcome;
    // on a timeout the phase stays, so the drain below waits on the same one)
    auto sync_mma = [&](int sl) -> bool {
        const bool ok = wait_bounded(smem_u32(&bar[sl]), phase_s[sl]);
        const bool all = __syncthreads_and(ok) != 0;
        if (all) phase_s[sl] ^= 1u;
        fence_after();
        return all;
    };

    // epilogue of slot sl's layer: this thread's accumulator row of each M block
    auto epilogue = [&](int sl, int layer) {
        const uint32_t td = tmem + lane_off + (uint32_t)(sl * 128);
        if (layer < 3) {
            const float* bias = sBias + 32 * layer;
            unsigned char* dst = sm + kOffAct + sl * kActBytes;  // in place
#pragma unroll 1
            for (int m = 0; m < 3; ++m) {
                const int q = 128 * m + t, P = q + kPlane;
                const int R = P / kPlane, Cc = P - R * kPlane;
                const bool valid = q < 288 && Cc >= 1 && Cc <= 16;
                float v[32];
                tmem_ld32(td + m * 32, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = valid ? fmaxf(v[i] + bias[i], 0.0f) : 0.0f;
                store_pos(dst, kChunkA, P + 1, v);
            }
        } else {
            const float* sD = reinterpret_cast<const float*>(sm + kOffTile + sl * kTileBytes);
            const float* sG = sD + 256;
            const long long tile = tile_s[sl];
            const float sd = scale_s[sl];
#pragma unroll 1
            for (int m = 0; m < 3; ++m) {
                const int q = 128 * m + t, P = q + kPlane;
                const int R = P / kPlane, Cc = P - R * kPlane;
                float v[32];
                tmem_ld32(td + m * 16, v);  // columns 0..15 used (+16 unused)
                if (q < 288 && Cc >= 1 && Cc <= 16) {
                    const int px = (R - 1) * 16 + (Cc - 1);
                    const float y = v[0] + sBias[96];
                    const float d = sD[px], g = sG[px];
                    const float lo = kStartFrac * fmaxf(d + g, 1e-3f) - g;
                    u0[tile * 256 + px] = fmaxf(fmaf(sd, y, d), lo);
                }
            }
        }
    };

    // ---- start: each slot's first tile -------------------------------------
#pragma unroll
    for (int sl = 0; sl < kSlots; ++sl) {
        tile_s[sl] = (long long)blockIdx.x + (long long)sl * gridDim.x;
        scale_s[sl] = 1.0f;
        if (tile_s[sl] < src.n_tiles) gather(tile_s[sl], dv[sl], gv[sl]);
    }
#pragma unroll
    for (int sl = 0; sl < kSlots; ++sl) {
        if (tile_s[sl] >= src.n_tiles) continue;
        build(sl);
        issue(sl, 0);
        if (tile_s[sl] + stride < src.n_tiles) gather(tile_s[sl] + stride, dv[sl], gv[sl]);
    }

    // ---- alternate between the slots until both run out of tiles ------------
    for (;;) {
        bool any = false;
#pragma unroll
        for (int sl = 0; sl < kSlots; ++sl) {
            if (!alive || tile_s[sl] >= src.n_tiles) continue;
            any = true;
            if (!sync_mma(sl)) {
                alive = false;
                break;
            }
            epilogue(sl, layer_s[sl]);
            if (layer_s[sl] < 3) {
                ++layer_s[sl];
                issue(sl, layer_s[sl]);
            } else {
                // tile done: its successor's pixels were gathered during its layers
                tile_s[sl] += stride;
                layer_s[sl] = 0;
                if (tile_s[sl] < src.n_tiles) {
                    build(sl);
                    issue(sl, 0);
                    if (tile_s[sl] + stride < src.n_tiles)
                        gather(tile_s[sl] + stride, dv[sl], gv[sl]);
                }
            }
        }
        if (!any || !alive) break;
    }

    if (!alive) {
        if (t == 0 && status) atomicExch(status, 1);
        // drain: give every slot's outstanding MMAs a bounded time to complete
#pragma unroll
        for (int sl = 0; sl < kSlots; ++sl)
            if (tile_s[sl] < src.n_tiles) wait_bounded(smem_u32(&bar[sl]), phase_s[sl]);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols)
                     : "memory");
    }
}

int launch(const Src& src, const float* params, float* u0, int32_t* status, cudaStream_t s) {
    if (cudaFuncSetAttribute(infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) !=
        cudaSuccess)
        return NCSB_ECUDA;
    // all of the unified L1 as shared memory, so two CTAs fit on an SM
    cudaFuncSetAttribute(infer_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    int dev = 0, sms = 1;
    if (cudaGetDevice(&dev) != cudaSuccess) return NCSB_ECUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // CTAs per SM from the shared-memory budget (the occupancy query assumes the
    // default carveout); more CTAs than fit only queue, results do not change
    int per_sm_bytes = 0, reserved = 0;
    cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    int per_sm = per_sm_bytes / (kSmemBytes + 1024 + reserved);  // + static shared memory
    per_sm = per_sm < 1 ? 1 : (per_sm > 2 ? 2 : per_sm);
    long long grid = (long long)sms * per_sm;
    if (grid > (src.n_tiles + kSlots - 1) / kSlots) grid = (src.n_tiles + kSlots - 1) / kSlots;
    infer_tc<<<(unsigned)grid, kThreads, kSmemBytes, s>>>(src, params, u0, status);
    return cudaGetLastError() == cudaSuccess ? NCSB_OK : NCSB_ECUDA;
}

int launch_batch(const float* params, const StackDesc* stacks, int n_stacks, long long n_tiles,
                 float* u0, int32_t* status, cudaStream_t s) {
    if (n_tiles == 0) return NCSB_OK;
    Src src{};
    src.stacks = stacks;
    src.n_stacks = n_stacks;
    src.tiles_x = 1;
    src.tiles_y = 1;
    src.n_tiles = n_tiles;
    return launch(src, params, u0, status, s);
}

static_assert(2 * (kSmemBytes + 2048) <= 228 * 1024, "two CTAs per SM");
static_assert(2 * kTmemCols <= 512, "two CTAs' tensor memory fits an SM");
static_assert(kOffAct % 16 == 0 && kActBytes % 16 == 0 && kOffTile % 16 == 0, "alignment");
static_assert(kIm2colPos + kQ <= kPos - 21, "im2col rows stay inside the rewritten range");

}  // namespace nettc
}  // namespace ncsb

using namespace ncsb::nettc;
using ncsb::tiles_along;

extern "C" {

int ncsb_net_infer_stack_tc(const float* params, const float* images, int n_frames, int height,
                            int width, const float* gamma, int gamma_per_frame, float* u0,
                            int32_t* status, void* stream) {
    if (!params || !images || !gamma || !u0 || n_frames < 0 || height <= 0 || width <= 0)
        return NCSB_EINVAL;
    if (height < 14 || width < 14) return NCSB_ESIZE;
    if (n_frames == 0) return NCSB_OK;
    Src src{};
    src.d = images;
    src.gamma = gamma;
    src.gamma_frame_stride = gamma_per_frame ? (long long)height * width : 0;
    src.H = height;
    src.W = width;
    src.tiles_x = tiles_along(height);
    src.tiles_y = tiles_along(width);
    src.n_tiles = (long long)n_frames * src.tiles_x * src.tiles_y;
    return launch(src, params, u0, status, (cudaStream_t)stream);
}

int ncsb_net_infer_tiles_tc(const float* params, const float* d, const float* gamma,
                            int64_t n_tiles, float* u0, int32_t* status, void* stream) {
    if (!params || !d || !gamma || !u0 || n_tiles < 0) return NCSB_EINVAL;
    if (n_tiles == 0) return NCSB_OK;
    Src src{};
    src.tile_mode = 1;
    src.d = d;
    src.gamma = gamma;
    src.tiles_x = 1;
    src.tiles_y = 1;
    src.H = 16;
    src.W = 16;
    src.n_tiles = n_tiles;
    return launch(src, params, u0, status, (cudaStream_t)stream);
}

}  // extern "C"
