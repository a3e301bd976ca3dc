// ncs_tc.cu -- the tensor-core form (NCSB_MODE_TC_TF32, NCSB_MODE_TC_BF16X3):
// the spectral-preconditioned L-BFGS of ncs_spectral.cu with every 16x16
// Fourier transform done by the 5th-generation tensor cores (tcgen05).
//
// The noise term is the quadratic form alpha u'Q u, Q = (1/256) F^H diag(M^2) F
// (clib/pyCNCS/ncs.c:220-299, cuda/ncs.cu:743-817).  Each solver pass
// applies one operator of the form (1/256) F^H diag(h) F to one vector per
// tile: h = 2 alpha M^2 gives v = 2 alpha Q u at the start, and
// h = 1 / (lambda + 2 alpha M^2) gives p = H0 q in an iteration (the
// spectral initial inverse Hessian; 2 alpha Q H0 q = q - lambda H0 q needs no
// transform of its own, nor does any line-search trial).  Here that operator
// is four GEMMs over the tiles of a CTA (M = 16 rows per tile, 4 tiles):
//   1. row DFT, real -> packed half spectrum:    [x]      (K 16)  x B1 (N 16)
//   2. column DFT, complex, per column 0..8:     [Y^T]    (K 32)  x B2 (N 32)
//      then the weights h, elementwise
//   3. inverse column DFT:                        [hZ]     (K 32)  x B3 (N 32)
//   4. inverse row DFT, packed -> real:           [W]      (K 18, padded to 32) x B4 (N 16)
// Stage 1 sees each tile as 16 rows x 16 columns; stages 2 and 3 as one row
// per column frequency kc = 0..8 (rows 9..15 are padding whose results are
// never read) holding the real and imaginary parts over 16 rows; stage 4 as
// 16 rows again.  The transposes between them happen in the epilogues: each
// warp reads its tile's 16 accumulator lanes from tensor memory
// (tcgen05.ld.16x256b: lane L gets rows L/4 and L/4 + 8), which is exactly
// the warp solvers' lane layout (rows P, P + 8, columns Qd + 4j), and writes
// the next stage's K-major operand.  The orders of K and N in the constant
// matrices B1..B4 are chosen so that every lane writes runs of 2, 4 or 8
// consecutive K values (vector stores, no shuffles).  The weights are applied
// in registers between stages 2 and 3.
//
// Precision: TF32 operands (rounded to nearest when written; 10-bit
// mantissa, so each transform carries about 1e-3 relative error) with FP32
// accumulation, or a three-way BF16 split (hi/lo of both operands,
// hi*hi + lo*hi + hi*lo, about 1e-5), FP32 accumulation.  The
// line-search cost differences, the Armijo test and the convergence test are
// those of the spectral form: the directional model f(u + tp) - f(u) =
// dLL + t p'v + t^2/2 p'w (FP64 across the warp) is consistent with the
// gradient g = gLL + v by construction, whatever the transform's rounding,
// which only perturbs v = 2 alpha Q u (kept by updates v += t w) and the
// preconditioner.  The final per-tile cost reported is the model's; callers
// that want the exact cost of the result evaluate it from u.
//
// Lock step: the warps of a CTA each own a tile and pass through the
// four stages together (one CTA barrier before each stage's MMAs; thread 0
// issues them and commits to an mbarrier all threads wait on, suspended
// rather than spinning).  A warp whose
// tile finishes takes the next one from the work queue at the start of the
// next pass, so every pass carries a full set of tiles until the queue runs
// dry.
// Waits are bounded: a wait that runs out sets a.flag, every thread leaves
// the pass loop at the next barrier, the outstanding MMAs get a bounded wait
// and tensor memory is freed.
#include "ncs_warp_common.cuh"
#include "tc_sm100.cuh"

namespace ncsb {

using namespace warp;

namespace tcs {

// Tiles (warps) per CTA: the GEMMs have M = 16 kTiles rows.  With 4 tiles
// (M = 64) four CTAs share an SM, and the tensor core writes a CTA's 64
// accumulator rows to lanes 0-15 of each 32-lane quarter of tensor memory,
// rows 16 w .. 16 w + 15 to the quarter of warp w -- so each warp reads its
// own tile.  (With 8 tiles, M = 128 and two CTAs per SM, row m is lane m.)
constexpr int kTiles = 4;
constexpr int kM = 16 * kTiles;
constexpr int kTcWarps = kTiles;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr int kMinBlocks = 16 / kTiles;  // 128 registers a thread fill the register file
// D of stages 1 and 3 at column 0, of stages 2 and 4 at column 32: a stage's
// accumulators are read before the MMAs of the stage after next are issued
constexpr uint32_t kTmemCols = 64;
constexpr long long kWaitTries = 1ll << 17;  // mbarrier polls of <= 20 us before giving up
constexpr long long kSpinTries = 1ll << 26;  // mbarrier polls without suspending (seconds)

// Operand A (kM rows): groups of 8 rows, 128 B apart; K chunks (16 bytes of
// K per row) kALbo apart.  The extra 16 bytes move consecutive chunks to the
// next 16-byte bank group, so the epilogue stores of a warp (lanes spread
// over chunks and rows) spread over all banks.
constexpr int kALbo = (kM / 8) * 128 + 16;

// Shared-memory plan for element size ES (4: TF32, 2: BF16) and parts NP
// (1: TF32, 2: BF16 hi and lo).
template <bool BF>
struct Plan {
    static constexpr int ES = BF ? 2 : 4;
    static constexpr int NP = BF ? 2 : 1;
    static constexpr int KPC = 16 / ES;                 // K values per 16-byte core row
    static constexpr int B1 = 16 * 16 * ES;             // N 16 x K 16
    static constexpr int B2 = 32 * 32 * ES;             // N 32 x K 32
    static constexpr int B4 = 16 * 32 * ES;             // N 16 x K 32
    static constexpr int BPART = B1 + 2 * B2 + B4;      // one part of B1..B4
    static constexpr int OFF_B = 0;
    static constexpr int A1 = (16 / KPC) * kALbo;       // stage-1 operand (K 16), one part
    static constexpr int A2 = (32 / KPC) * kALbo;       // stages 2-4 operand (K 32), one part
    static constexpr int OFF_A1 = OFF_B + NP * BPART;
    static constexpr int OFF_A2 = OFF_A1 + NP * A1;
    // per warp: s, y, Q s (1 KB each), then the pixel terms c, gamma (2 KB)
    static constexpr int OFF_HIST = OFF_A2 + NP * A2;
    static constexpr int BYTES = OFF_HIST + kTcWarps * 5 * 1024;
};

// Byte offset of element (row, k) of a K-major operand whose 8-row groups
// are 128 B apart and whose K chunks are `lbo` apart.
template <int ES>
__device__ __forceinline__ int koff(int row, int k, int lbo) {
    constexpr int KPC = 16 / ES;
    return (k / KPC) * lbo + (row >> 3) * 128 + (row & 7) * 16 + (k % KPC) * ES;
}

// FP32 -> TF32 rounded to nearest (ties away from zero); the tensor core
// itself would drop the low 13 mantissa bits (round toward zero), which biases
// every product by about -2^-11 relative.
__device__ __forceinline__ float tf32r(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ uint32_t bf2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
// hi = bf16(a), lo = bf16(a - hi), for a pair
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = bf2(a - hf.x, b - hf.y);
}

// Operand stores: 2, 4 or 8 consecutive K values of one row, k0 aligned to the run.
template <bool BF>
__device__ __forceinline__ void st2(unsigned char* buf, int part_bytes, int row, int k0,
                                    float x0, float x1) {
    const int o = koff<Plan<BF>::ES>(row, k0, kALbo);
    if constexpr (BF) {
        uint32_t hi, lo;
        split2(x0, x1, hi, lo);
        *reinterpret_cast<uint32_t*>(buf + o) = hi;
        *reinterpret_cast<uint32_t*>(buf + part_bytes + o) = lo;
    } else {
        *reinterpret_cast<float2*>(buf + o) = make_float2(tf32r(x0), tf32r(x1));
    }
}
template <bool BF>
__device__ __forceinline__ void st4(unsigned char* buf, int part_bytes, int row, int k0, float x0,
                                    float x1, float x2, float x3) {
    const int o = koff<Plan<BF>::ES>(row, k0, kALbo);
    if constexpr (BF) {
        uint32_t h0, l0, h1, l1;
        split2(x0, x1, h0, l0);
        split2(x2, x3, h1, l1);
        *reinterpret_cast<uint2*>(buf + o) = make_uint2(h0, h1);
        *reinterpret_cast<uint2*>(buf + part_bytes + o) = make_uint2(l0, l1);
    } else {
        *reinterpret_cast<float4*>(buf + o) =
            make_float4(tf32r(x0), tf32r(x1), tf32r(x2), tf32r(x3));
    }
}
template <bool BF>
__device__ __forceinline__ void st8(unsigned char* buf, int part_bytes, int row, int k0,
                                    const float (&x)[8]) {
    if constexpr (BF) {
        const int o = koff<2>(row, k0, kALbo);
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) split2(x[2 * i], x[2 * i + 1], h[i], l[i]);
        *reinterpret_cast<uint4*>(buf + o) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(buf + part_bytes + o) = make_uint4(l[0], l[1], l[2], l[3]);
    } else {
        *reinterpret_cast<float4*>(buf + koff<4>(row, k0, kALbo)) =
            make_float4(tf32r(x[0]), tf32r(x[1]), tf32r(x[2]), tf32r(x[3]));
        *reinterpret_cast<float4*>(buf + koff<4>(row, k0 + 4, kALbo)) =
            make_float4(tf32r(x[4]), tf32r(x[5]), tf32r(x[6]), tf32r(x[7]));
    }
}

// Entries of the constant matrices, B[n][k] (row n = output column of the stage).
__device__ float b_entry(int which, int n, int k) {
    float sn, cs;
    if (which == 1) {  // row DFT: k -> pixel column c; n -> (slot, re/im)
        const int c = (k >> 2) + 4 * (k & 3), slot = n >> 1, ri = n & 1;
        if (slot == 0) return ri == 0 ? 1.0f : ((c & 1) ? -1.0f : 1.0f);  // Re X0, Re X8
        sincospif((float)((slot * c) & 15) / 8.0f, &sn, &cs);
        return ri == 0 ? cs : -sn;
    }
    if (which == 2) {  // column DFT: k -> (row r, re/im in), n -> (re/im out, kr)
        const int ro = n & 1, kr = n >> 1;
        const int r = (k >> 2) + 8 * ((k >> 1) & 1), ri = k & 1;
        sincospif((float)((kr * r) & 15) / 8.0f, &sn, &cs);
        if (ro == 0) return ri == 0 ? cs : sn;
        return ri == 0 ? -sn : cs;
    }
    if (which == 3) {  // inverse column DFT / 16: k -> (kr, re/im in), n -> (re/im out, r)
        const int ro = n & 1, r = n >> 1;
        const int kr = 4 * ((k & 7) >> 1) + (k >> 3), ri = k & 1;
        sincospif((float)((kr * r) & 15) / 8.0f, &sn, &cs);
        const float s16 = 1.0f / 16.0f;
        if (ro == 0) return ri == 0 ? cs * s16 : -sn * s16;
        return ri == 0 ? sn * s16 : cs * s16;
    }
    // inverse row DFT / 16, packed -> real: k = 2 kc + re/im (k < 18), n -> column c
    const int c = ((n & 7) >> 1) + 4 * (n & 1) + 8 * (n >> 3);
    const int kc = k >> 1, ri = k & 1;
    if (k >= 18 || ri == 1 && (kc == 0 || kc == 8)) return 0.0f;
    if (kc == 0) return 1.0f / 16.0f;
    if (kc == 8) return ((c & 1) ? -1.0f : 1.0f) / 16.0f;
    sincospif((float)((kc * c) & 15) / 8.0f, &sn, &cs);
    return ri == 0 ? 2.0f * cs / 16.0f : -2.0f * sn / 16.0f;
}

// Write one constant matrix (N rows x K) in its K-major layout, all parts.
template <bool BF>
__device__ void build_b(unsigned char* base, int which, int N, int K) {
    constexpr int ES = Plan<BF>::ES;
    const int lbo = N * 16;
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) {
        const int n = i / K, k = i - n * K;
        const float v = b_entry(which, n, k);
        const int o = koff<ES>(n, k, lbo);
        if constexpr (BF) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
            *reinterpret_cast<__nv_bfloat16*>(base + o) = h;
            *reinterpret_cast<__nv_bfloat16*>(base + Plan<BF>::BPART + o) = l;
        } else {
            *reinterpret_cast<float*>(base + o) = tf32r(v);
        }
    }
}

// Thread 0: the MMAs of one stage into tensor memory column `col`.
template <bool BF>
__device__ __forceinline__ void issue_stage(int stage, uint32_t tmem, uint32_t sb, uint32_t sa1,
                                            uint32_t sa2) {
    using PL = Plan<BF>;
    const int N = (stage == 1 || stage == 4) ? 16 : 32;
    const uint32_t lbo_b = (uint32_t)N * 16;
    const uint32_t boff = stage == 1 ? 0 : (stage == 2 ? PL::B1 : (stage == 3 ? PL::B1 + PL::B2
                                                                            : PL::B1 + 2 * PL::B2));
    const uint32_t a = stage == 1 ? sa1 : sa2;
    const uint32_t apart = stage == 1 ? PL::A1 : PL::A2;
    const uint32_t col = (uint32_t)((stage - 1) & 1) * 32;
    // K steps of 2 chunks (TF32: K 8; BF16: K 16) -- stage 4 only up to K 24 / 32
    const int steps = BF ? (stage == 1 ? 1 : 2) : (stage == 1 ? 2 : (stage == 4 ? 3 : 4));
    for (int s = 0; s < steps; ++s) {
        const uint64_t ad = tc::sdesc(a + 2 * s * kALbo, kALbo, 128);
        const uint64_t bd = tc::sdesc(sb + boff + 2 * s * lbo_b, lbo_b, 128);
        if constexpr (BF) {
            const uint32_t id = tc::idesc_bf16(kM, N);
            const uint64_t adl = tc::sdesc(a + apart + 2 * s * kALbo, kALbo, 128);
            const uint64_t bdl = tc::sdesc(sb + PL::BPART + boff + 2 * s * lbo_b, lbo_b, 128);
            tc::mma_bf16(tmem + col, ad, bd, id, s > 0);  // hi x hi
            tc::mma_bf16(tmem + col, adl, bd, id, 1u);    // lo x hi
            tc::mma_bf16(tmem + col, ad, bdl, id, 1u);    // hi x lo
        } else {
            tc::mma_tf32(tmem + col, ad, bd, tc::idesc_tf32(kM, N), s > 0);
        }
    }
}

// Per-stack geometry of a single-stack launch.
struct Geo {
    const float* data;
    const float* gamma;
    float* out;
    long long gstride;
    int H, W, tiles_x, tiles_y;
};

}  // namespace tcs

using namespace tcs;

// Batch: tiles of several stacks (own shape, alpha and mask each, a.stacks)
// in one queue; a warp finds its tile's stack by binary search over the
// stacks' first tiles and keeps the descriptor in a shared slot.
template <bool BF, bool Warm, bool Batch>
__global__ void __launch_bounds__(kTcThreads, kMinBlocks) ncs_tc_kernel(const SolveArgs a) {
    using PL = Plan<BF>;
    extern __shared__ __align__(1024) unsigned char dsm[];
    __shared__ StackDesc s_stack[kTcWarps];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const float eps2 = a.eps * a.eps;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int P = lane >> 2, Qd = lane & 3;
    // the warp's tile slot: M rows 16 ts .. 16 ts + 15, in tensor-memory lanes
    // tl .. tl + 15 of the warp's quarter
    const int ts = kTiles == 8 ? 2 * (wid & 3) + (wid >> 2) : wid;
    const int row0 = 16 * ts;
    const int tl = kTiles == 8 ? row0 : 32 * wid;
    unsigned char* sB = dsm + PL::OFF_B;
    unsigned char* sA1 = dsm + PL::OFF_A1;
    unsigned char* sA2 = dsm + PL::OFF_A2;
    float4* hs = reinterpret_cast<float4*>(dsm + PL::OFF_HIST + wid * 5 * 1024);
    float4* hy = hs + 64;
    float4* hq = hy + 64;
    float4* terms = hq + 64;  // c and gamma, see load_terms

    // ---- set-up: constant matrices, zeroed operands, mbarrier, tensor memory
    build_b<BF>(sB, 1, 16, 16);
    build_b<BF>(sB + PL::B1, 2, 32, 32);
    build_b<BF>(sB + PL::B1 + PL::B2, 3, 32, 32);
    build_b<BF>(sB + PL::B1 + 2 * PL::B2, 4, 16, 32);
    for (int i = threadIdx.x; i < PL::NP * (PL::A1 + PL::A2) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sA1)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (threadIdx.x == 0) {
        tc::mbar_init(tc::smem_u32(&s_bar), 1);
        s_abort = 0;
    }
    if (wid == 0) tc::tmem_alloc(tc::smem_u32(&s_tmem), kTmemCols);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t tlane = tmem + ((uint32_t)tl << 16);
    const uint32_t sbu = tc::smem_u32(sB), sa1u = tc::smem_u32(sA1), sa2u = tc::smem_u32(sA2);
    const uint32_t bar = tc::smem_u32(&s_bar);
    uint32_t phase = 0;

    // M^2/256 at this lane's stage-2 bins: row kc = P at kr = 4q + Qd, and
    // (lanes with P = 0) row kc = 8.  A batch reads them per tile from its
    // stack's table in the spectral form's lane layout: bin (kr, kc) sits at
    // 8 (2 kc + kr % 2) + bitrev3(kr / 2).
    float mkA[4], mkB[4];
    auto load_bins = [&](const float* tab, bool lane_layout) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int kr = 4 * q + Qd;
            if (lane_layout) {
                mkA[q] = __ldg(tab + 8 * (2 * P + (kr & 1)) + bitrev3(kr >> 1));
                mkB[q] = __ldg(tab + 8 * (16 + (kr & 1)) + bitrev3(kr >> 1));
            } else {
                mkA[q] = __ldg(tab + kr * 16 + P);
                mkB[q] = __ldg(tab + kr * 16 + 8);
            }
        }
    };
    if (!Batch) load_bins(a.msq, false);
    float alpha = a.alpha, two_alpha = 2.0f * a.alpha, a512 = 512.0f * a.alpha;
    // the warp's stack geometry: the launch's, or its current stack's
    auto geo = [&]() -> Geo {
        if constexpr (Batch) {
            const StackDesc& sd = s_stack[wid];
            return Geo{sd.data, sd.gamma, sd.out, sd.gamma_frame_stride, sd.H, sd.W, sd.tiles_x,
                       sd.tiles_y};
        } else {
            return Geo{a.data, a.gamma, a.out, a.gamma_frame_stride, a.H, a.W, a.tiles_x,
                       a.tiles_y};
        }
    };

    // One stage: everyone's operand rows are in shared memory; thread 0
    // issues the stage's MMAs; all wait for them.  False: abort.
    auto run_stage = [&](int stage) -> bool {
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        if (s_abort) return false;
        if (threadIdx.x == 0) {
            tc::fence_after();
            issue_stage<BF>(stage, tmem, sbu, sa1u, sa2u);
            tc::commit(bar);
        }
        // a polling wait: threads that sleep in the wait measured slower
        bool ok = false;
        for (long long i = 0; i < kSpinTries && !ok; ++i) ok = tc::try_wait(bar, phase);
        phase ^= 1u;
        if (!ok) {
            s_abort = 1;
            if (a.flag) atomicExch(a.flag, 1);
        }
        tc::fence_after();
        return true;
    };

    // ---- per-warp solver state (the spectral form's, m = 1) -----------------
    bool has_tile = false;
    long long tile = 0;
    float u[8], v[8], g[8], p[8], w[8];  // c and gamma: in shared memory (terms)
    float rho = 0.0f, al = 0.0f, sg_newest = 0.0f, lam = 1.0f;
    bool sg_fresh = false, first = true;
    int status = kUnstarted, iters = 0, evals = 1, k = 0, start_pass = 0, fell_back = 0;
    int f = 0, ox = 0, oy = 0, own_r = 0, own_c = 0;
    bool aborted = false;

    auto load_d = [&](float (&dst)[8]) {
        if (a.tile_mode) {
            const float* dt = a.data + tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    dst[2 * j + s] = __ldg(dt + (P + 8 * s) * kTile + Qd + 4 * j);
        } else {
            const Geo sg = geo();
            const float* img = sg.data + (long long)f * sg.H * sg.W;
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const long long row = clampi(ox + P + 8 * s - 1, 0, sg.H - 1);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    dst[2 * j + s] =
                        __ldg(img + row * sg.W + clampi(oy + Qd + 4 * j - 1, 0, sg.W - 1));
            }
        }
    };

    for (;;) {
        // ---- a warp without a tile takes the next one ------------------------
        if (!has_tile) {
            unsigned long long tk = 0;
            if (lane == 0) tk = atomicAdd(a.queue, 1ull);
            tile = (long long)__shfl_sync(kFull, tk, 0);
            if (tile < a.n_tiles) {
                has_tile = true;
                float d[8], gm[8];
                long long lt = tile;  // index of the tile within its stack
                if constexpr (Batch) {
                    int lo = 0, hi = a.n_stacks - 1;
                    while (lo < hi) {  // last stack whose first tile is <= tile
                        const int mid = (lo + hi + 1) >> 1;
                        if (__ldg(&a.stacks[mid].tile_begin) <= tile) lo = mid;
                        else hi = mid - 1;
                    }
                    __syncwarp();  // every lane is done with the previous descriptor
                    if (lane == 0) s_stack[wid] = a.stacks[lo];
                    __syncwarp();
                    lt = tile - s_stack[wid].tile_begin;
                    alpha = s_stack[wid].alpha;
                    two_alpha = 2.0f * alpha;
                    a512 = 512.0f * alpha;
                    load_bins(a.mk_lane + (size_t)lo * 256, true);
                }
                if (a.tile_mode) {
                    const long long base = tile * kPix;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int s = 0; s < 2; ++s) {
                            const int off = (P + 8 * s) * kTile + Qd + 4 * j;
                            d[2 * j + s] = __ldg(a.data + base + off);
                            gm[2 * j + s] = __ldg(a.gamma + base + off);
                            u[2 * j + s] = Warm ? __ldg(a.u0 + base + off) : d[2 * j + s];
                        }
                } else {
                    const Geo sg = geo();
                    const long long per_frame = (long long)sg.tiles_x * sg.tiles_y;
                    f = (int)(lt / per_frame);
                    const int rem = (int)(lt - (long long)f * per_frame);
                    const int ti = rem / sg.tiles_y, tj = rem - (rem / sg.tiles_y) * sg.tiles_y;
                    ox = tile_origin(ti, sg.H);
                    oy = tile_origin(tj, sg.W);
                    own_r = (ti + 1 < sg.tiles_x ? tile_origin(ti + 1, sg.H) : ox + 14) - ox;
                    own_c = (tj + 1 < sg.tiles_y ? tile_origin(tj + 1, sg.W) : oy + 14) - oy;
                    const float* img = sg.data + (long long)f * sg.H * sg.W;
                    const float* gmap = sg.gamma + (long long)f * sg.gstride;
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const long long row = clampi(ox + P + 8 * s - 1, 0, sg.H - 1);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int col = clampi(oy + Qd + 4 * j - 1, 0, sg.W - 1);
                            d[2 * j + s] = __ldg(img + row * sg.W + col);
                            gm[2 * j + s] = __ldg(gmap + row * sg.W + col);
                            u[2 * j + s] = d[2 * j + s];
                        }
                    }
                    if (Warm) {
                        const float* ut = a.u0 + tile * kPix;
#pragma unroll
                        for (int j = 0; j < 4; ++j)
#pragma unroll
                            for (int s = 0; s < 2; ++s)
                                u[2 * j + s] = __ldg(ut + (P + 8 * s) * kTile + Qd + 4 * j);
                    }
                }
                __syncwarp();  // the previous tile's terms are no longer read
                store_terms(terms, lane, d, gm);
                __syncwarp();
                rho = al = sg_newest = 0.0f;
                lam = 1.0f;
                sg_fresh = false;
                first = true;
                status = kUnstarted;
                iters = 0;
                evals = 1;
                k = 0;
                start_pass = Warm ? 2 : 0;
                fell_back = 0;
            }
        }
        if (!__syncthreads_or(has_tile ? 1 : 0) || s_abort) break;

        // ---- pre-transform: the vector to transform ----------------------------
        float q[8];
        if (has_tile) {
            if (first) {
                if (start_pass == 1) {
                    load_d(q);
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i) q[i] = u[i];
                }
            } else {
                // two-loop, first half (m = 1)
#pragma unroll
                for (int i = 0; i < 8; ++i) q[i] = -g[i];
                if (k > 0) {
                    float hv[8];
                    float dot;
                    if (sg_fresh) {
                        dot = -sg_newest;  // q = -g here
                    } else {
                        load_hist(hs, lane, hv);
                        float acc = 0.0f;
#pragma unroll
                        for (int e = 0; e < 8; ++e) acc = fmaf(hv[e], q[e], acc);
                        dot = warp_sum_f(acc);
                    }
                    al = rho * dot;
                    load_hist(hy, lane, hv);
#pragma unroll
                    for (int e = 0; e < 8; ++e) q[e] = fmaf(-al, hv[e], q[e]);
                }
            }
            // stage-1 operand: rows P, P + 8; K = 4 Qd + j holds column Qd + 4 j
#pragma unroll
            for (int s = 0; s < 2; ++s)
                st4<BF>(sA1, PL::A1, row0 + P + 8 * s, 4 * Qd, q[s], q[2 + s], q[4 + s],
                        q[6 + s]);
        }

        // ---- the transform: four GEMM stages -----------------------------------
        if (!run_stage(1)) break;
        if (has_tile) {
            float e[8];
            tc::tmem_ld_16x256b_x2(tlane + 0, e);
            tc::tmem_wait_ld();
            // slots Qd and Qd + 4 of rows P, P + 8: (Re, Im) of row frequency
            // kc = slot, slot 0 = (Re X0, Re X8); stage-2 K = 4 r' + 2 half + re/im
            if (Qd == 0) {
                st4<BF>(sA2, PL::A2, row0 + 0, 4 * P, e[0], 0.0f, e[2], 0.0f);
                st4<BF>(sA2, PL::A2, row0 + 8, 4 * P, e[1], 0.0f, e[3], 0.0f);
            } else {
                st4<BF>(sA2, PL::A2, row0 + Qd, 4 * P, e[0], e[1], e[2], e[3]);
            }
            st4<BF>(sA2, PL::A2, row0 + Qd + 4, 4 * P, e[4], e[5], e[6], e[7]);
        }
        if (!run_stage(2)) break;
        if (has_tile) {
            float e[16];
            tc::tmem_ld_16x256b_x4(tlane + 32, e);
            tc::tmem_wait_ld();
            // weights at (kr = 4 q + Qd, kc = P) and, for P = 0, kc = 8
            float r0[8], r8[8];
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const float hA = first ? a512 * mkA[qq] : rcp_fast(fmaf(a512, mkA[qq], lam));
                const float hB = first ? a512 * mkB[qq] : rcp_fast(fmaf(a512, mkB[qq], lam));
                r0[2 * qq] = e[4 * qq] * hA;
                r0[2 * qq + 1] = e[4 * qq + 1] * hA;
                r8[2 * qq] = e[4 * qq + 2] * hB;
                r8[2 * qq + 1] = e[4 * qq + 3] * hB;
            }
            st8<BF>(sA2, PL::A2, row0 + P, 8 * Qd, r0);
            if (P == 0) st8<BF>(sA2, PL::A2, row0 + 8, 8 * Qd, r8);
        }
        if (!run_stage(3)) break;
        if (has_tile) {
            float e[16];
            tc::tmem_ld_16x256b_x4(tlane + 0, e);
            tc::tmem_wait_ld();
            // (Re, Im) of W[r][kc] for r = 4 q + Qd, kc = P (and 8): stage-4 row r, K = 2 kc
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                st2<BF>(sA2, PL::A2, row0 + 4 * qq + Qd, 2 * P, e[4 * qq], e[4 * qq + 1]);
                if (P == 0)
                    st2<BF>(sA2, PL::A2, row0 + 4 * qq + Qd, 16, e[4 * qq + 2], e[4 * qq + 3]);
            }
        }
        if (!run_stage(4)) break;
        if (has_tile) {
            float e[8];
            tc::tmem_ld_16x256b_x2(tlane + 32, e);
            tc::tmem_wait_ld();
            p[0] = e[0]; p[1] = e[2]; p[2] = e[1]; p[3] = e[3];
            p[4] = e[4]; p[5] = e[6]; p[6] = e[5]; p[7] = e[7];
        }
        tc::fence_before();  // this pass's tensor-memory loads precede the next stage's MMAs
        if (!has_tile) continue;

        // ---- post-transform: the spectral form's pass, from p -------------------
        bool done = false;
        if (!first) {  // w = 2 alpha Q H0 q = q - lambda H0 q
            if (two_alpha > 0.0f) {
#pragma unroll
                for (int i = 0; i < 8; ++i) w[i] = fmaf(-lam, p[i], q[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) w[i] = 0.0f;
            }
        }
        if (first) {
            bool init = true;
            if (start_pass == 2) {
                // the spectral form's bound: f(u0) - f(d) <= LL(u0) - LL(d) +
                // (u0 - d)'v0, v0 = 2 alpha Q u0 = p; accept u0 when <= 0,
                // else transform d next for the exact comparison
                float dd[8], c[8], gm[8];
                load_d(dd);
                load_terms(terms, lane, c, gm);
                float dl = 0.0f, dq = 0.0f;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float lr = __fsub_rn(__logf(fmaxf(u[i] + gm[i], kFitMin)),
                                               __logf(fmaxf(dd[i] + gm[i], kFitMin)));
                    dl += fmaf(-c[i], lr, u[i] - dd[i]);
                    dq += __fmul_rn(__fsub_rn(u[i], dd[i]), p[i]);
                }
                const double bound = warp_sum_d((double)dl + (double)dq);
                if (bound <= 0.0) {
                    start_pass = 0;
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i) w[i] = p[i];
                    start_pass = 1;
                    init = false;
                }
            } else if (start_pass == 1) {
                float dd[8], c[8], gm[8];
                load_d(dd);
                load_terms(terms, lane, c, gm);
                float dl = 0.0f, dq = 0.0f;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float lr = __fsub_rn(__logf(fmaxf(u[i] + gm[i], kFitMin)),
                                               __logf(fmaxf(dd[i] + gm[i], kFitMin)));
                    dl += fmaf(-c[i], lr, u[i] - dd[i]);
                    dq += __fsub_rn(__fmul_rn(u[i], w[i]), __fmul_rn(dd[i], p[i]));
                }
                const double delta = warp_sum_d((double)dl + 0.5 * (double)dq);
                if (delta <= 0.0) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) p[i] = w[i];
                } else {
                    fell_back = 1;
#pragma unroll
                    for (int i = 0; i < 8; ++i) u[i] = dd[i];
                }
                start_pass = 0;
            }
            if (init) {
                first = false;
                float c[8], gm[8];
                load_terms(terms, lane, c, gm);
                float uu = 0.0f, gg = 0.0f, ll = 0.0f;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    v[i] = p[i];
                    const float ia = rcp_fast(fmaxf(u[i] + gm[i], kFitMin));
                    const float r = c[i] * ia;
                    g[i] = 1.0f - r + v[i];
                    uu = fmaf(u[i], u[i], uu);
                    gg = fmaf(g[i], g[i], gg);
                    ll = fmaf(r, ia, ll);
                }
                uu = warp_sum_f(uu);
                gg = warp_sum_f(gg);
                lam = warp_sum_f(ll) * (1.0f / 256.0f);
                if (gg <= eps2 * fmaxf(uu, 1.0f)) {
                    status = kSuccess;
                    done = true;
                }
            }
        } else {
            // two-loop, second half: p += coef s, w += coef Q s
            if (k > 0) {
                float hv[8];
                load_hist(hy, lane, hv);
                float acc = 0.0f;
#pragma unroll
                for (int e2 = 0; e2 < 8; ++e2) acc = fmaf(hv[e2], p[e2], acc);
                const float coef = al - rho * warp_sum_f(acc);
                load_hist(hs, lane, hv);
#pragma unroll
                for (int e2 = 0; e2 < 8; ++e2) p[e2] = fmaf(coef, hv[e2], p[e2]);
                load_hist(hq, lane, hv);
#pragma unroll
                for (int e2 = 0; e2 < 8; ++e2) w[e2] = fmaf(coef, hv[e2], w[e2]);
            }
            // this lane's part of the cost change at step t, and whether a pixel
            // crosses the barrier fraction
            // (pixels 2j and 2j + 1, rows P and P + 8, as packed FP32 pairs)
            auto trial_part = [&](float t, float& part, bool& cross) {
                float c[8], gm[8];
                load_terms(terms, lane, c, gm);
                const float2 t2 = splat(t);
                float term = 0.0f;
                cross = false;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // log(max(ni, F)) - log(max(ai, F)) = log1p((max(ni, F) - A) / A),
                    // A = max(ai, F); above the floor the numerator is the exact
                    // step tp (branch free: one select instead of a branch)
                    const float2 ai = pair(u, j) + pair(gm, j);
                    const float2 tp = t2 * pair(p, j);
                    const float2 ni = ai + tp;
                    const float2 bar = splat(kBarrierFrac) * ai;
                    float2 num, rA;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float a1 = h ? ai.y : ai.x, n1 = h ? ni.y : ni.x;
                        const bool in_dom = a1 >= kFitMin && n1 >= kFitMin;
                        const float A = fmaxf(a1, kFitMin);
                        (h ? num.y : num.x) = in_dom ? (h ? tp.y : tp.x) : fmaxf(n1, kFitMin) - A;
                        (h ? rA.y : rA.x) = rcp_fast(A);
                        cross |= (a1 >= kFitMin) && (n1 < (h ? bar.y : bar.x));
                    }
                    const float2 l = log1p_ls(num * rA);
                    term += fmaf(-c[2 * j], l.x, tp.x);
                    term += fmaf(-c[2 * j + 1], l.y, tp.y);
                }
                part = term;
            };
            // the slopes and the first trial's (t = 1) cost change in one FP64
            // reduction: the trial depends on p alone and is almost always accepted
            float gp = 0.0f, pv = 0.0f, pw = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                gp = fmaf(g[i], p[i], gp);
                pv = fmaf(p[i], v[i], pv);
                pw = fmaf(p[i], w[i], pw);
            }
            float part0;
            bool cross0;
            trial_part(1.0f, part0, cross0);
            const bool any_cross0 = __any_sync(kFull, cross0);
            double gd = (double)gp, dpv = (double)pv, dpw = (double)pw, dl0 = (double)part0;
            warp_sum4_d(gd, dpv, dpw, dl0, lane);
            if (!(gd < 0.0)) {
                // not a descent direction: drop the history, or fail without one
                if (k == 0) {
                    status = kIncreasingGradient;
                    done = true;
                } else {
                    k = 0;
                    sg_fresh = false;
                }
            } else {
                float t = 1.0f;
                bool ok = false;
                for (int trial = 0; trial < 64; ++trial) {
                    double dl = dl0;
                    bool any_cross = any_cross0;
                    if (trial > 0) {
                        float part;
                        bool cross;
                        trial_part(t, part, cross);
                        any_cross = __any_sync(kFull, cross);
                        dl = warp_sum_d((double)part);
                    }
                    ++evals;
                    const double td = (double)t;
                    const double delta =
                        any_cross ? CUDART_INF : dl + td * dpv + 0.5 * td * td * dpw;
                    if (delta <= (double)a.c1 * td * gd) {
                        ok = true;
                        break;
                    }
                    t *= 0.5f;
                    if (!(t >= a.min_step)) break;  // also stops on NaN
                }
                if (!ok) {
                    status = kMinimumStep;
                    done = true;
                } else {
                    // accept; new pair (s, y, Q s = t w)
                    float s[8], y[8], c[8], gm[8];
                    load_terms(terms, lane, c, gm);
                    const float2 t2 = splat(t), z2 = make_float2(0.0f, 0.0f);
                    float2 sy2 = z2, uu2 = z2, gg2 = z2, ll2 = z2, mv2 = z2, sg2 = z2;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {  // pixel pairs, packed FP32
                        const float2 uj = pair(u, j);
                        const float2 un = fma2(t2, pair(p, j), uj);
                        const float2 wj = pair(w, j) * t2;
                        const float2 vj = pair(v, j) + wj;
                        const float2 A = un + pair(gm, j);
                        const float2 ia = make_float2(rcp_fast(fmaxf(A.x, kFitMin)),
                                                      rcp_fast(fmaxf(A.y, kFitMin)));
                        const float2 r = pair(c, j) * ia;
                        const float2 gn = (splat(1.0f) - r) + vj;
                        const float2 sj = un - uj, yj = gn - pair(g, j);
                        // mv = s's squared norm: zero when no pixel moved (steps below about
                        // 1e-22, whose squares underflow, count as none)
                        mv2 = fma2(sj, sj, mv2);
                        sy2 = fma2(sj, yj, sy2);
                        sg2 = fma2(sj, gn, sg2);
                        uu2 = fma2(un, un, uu2);
                        gg2 = fma2(gn, gn, gg2);
                        ll2 = fma2(r, ia, ll2);
                        set_pair(w, j, wj);
                        set_pair(v, j, vj);
                        set_pair(s, j, sj);
                        set_pair(y, j, yj);
                        set_pair(u, j, un);
                        set_pair(g, j, gn);
                    }
                    float sy = sy2.x + sy2.y, uu = uu2.x + uu2.y, gg = gg2.x + gg2.y;
                    float ll = ll2.x + ll2.y, mv = mv2.x + mv2.y, sgv = sg2.x + sg2.y;
                    {
                        float vals[8] = {sy, uu, gg, ll, mv, sgv};
                        const float tot = warp_transpose_sum<8>(vals, lane);
                        sy = __shfl_sync(kFull, tot, 0);
                        uu = __shfl_sync(kFull, tot, 1);
                        gg = __shfl_sync(kFull, tot, 2);
                        ll = __shfl_sync(kFull, tot, 3);
                        mv = __shfl_sync(kFull, tot, 4);
                        sgv = __shfl_sync(kFull, tot, 5);
                    }
                    ++iters;
                    lam = ll * (1.0f / 256.0f);
                    if (gg <= eps2 * fmaxf(uu, 1.0f)) {
                        status = kSuccess;
                        done = true;
                    } else if (mv == 0.0f) {
                        status = kReachedMaxPrecision;
                        done = true;
                    } else {
                        sg_fresh = sy > 0.0f;
                        if (sy > 0.0f) {
                            sg_newest = sgv;
                            store_hist(hs, lane, s);
                            store_hist(hy, lane, y);
                            store_hist(hq, lane, w);
                            rho = rcp_fast(sy);
                            k = 1;
                        }
                    }
                }
            }
        }
        // the cap, checked where the next pass would begin
        if (!done && !first && iters >= a.max_iters) {
            status = kReachedMaxIters;
            done = true;
        }
        if (!done) continue;

        // ---- outputs -------------------------------------------------------------
        if (a.cost) {
            float c[8], gm[8];
            load_terms(terms, lane, c, gm);
            double e0 = 0.0, e1 = 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                e0 += (double)u[i] - (double)c[i] * log(fmax((double)u[i] + gm[i], 1.0e-6));
                e1 += (double)u[i] * v[i];
            }
            e0 = warp_sum_d(e0);
            e1 = warp_sum_d(e1);
            if (lane == 0) a.cost[tile] = e0 + 0.5 * e1;  // v = 2 alpha Q u (kept by updates)
        }
        if (lane == 0) {
            if (a.iters) a.iters[tile] = iters;
            if (a.status) a.status[tile] = status;
            if (a.evals) a.evals[tile] = evals;
            if (Warm && a.start) a.start[tile] = fell_back;
        }
        if (a.tile_mode) {
            const long long base = tile * kPix;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    a.out[base + (P + 8 * s) * kTile + Qd + 4 * j] = u[2 * j + s];
        } else {
            const Geo sg = geo();
            float* o = sg.out + (long long)f * sg.H * sg.W;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int cc = Qd + 4 * j;
                if (cc < 1 || cc > own_c) continue;
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int rr = P + 8 * s;
                    if (rr >= 1 && rr <= own_r)
                        o[(long long)(ox + rr - 1) * sg.W + oy + cc - 1] = u[2 * j + s];
                }
            }
        }
        has_tile = false;
    }
    (void)alpha;
    aborted = s_abort != 0;
    if (aborted) {
        // give the outstanding MMAs (the stage whose wait ran out) a bounded
        // time to complete before the tensor memory is freed
        tc::wait_bounded(bar, phase ^ 1u, kWaitTries);
    }
    tc::fence_before();
    __syncthreads();
    if (wid == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

namespace {

using TcKernel = void (*)(SolveArgs);

template <bool BF>
TcKernel tc_variant_p(bool warm, bool batch) {
    if (batch) return warm ? ncs_tc_kernel<BF, true, true> : ncs_tc_kernel<BF, false, true>;
    return warm ? ncs_tc_kernel<BF, true, false> : ncs_tc_kernel<BF, false, false>;
}

TcKernel tc_variant(bool bf16x3, bool warm, bool batch) {
    return bf16x3 ? tc_variant_p<true>(warm, batch) : tc_variant_p<false>(warm, batch);
}

size_t tc_smem_bytes(bool bf16x3) {
    return bf16x3 ? (size_t)Plan<true>::BYTES : (size_t)Plan<false>::BYTES;
}

}  // namespace

int tc_tiles_per_cta() { return kTiles; }

namespace {
cudaError_t prepare(TcKernel fn, size_t smem) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // all of the unified L1 as shared memory: two CTAs per SM need 2 x ~62 KB
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    return e;
}
}  // namespace

// Grid: CTAs of kTiles tiles, persistent over the work queue.
cudaError_t launch_tc(const SolveArgs& args, bool bf16x3, int grid, cudaStream_t stream) {
    const TcKernel fn = tc_variant(bf16x3, args.u0 != nullptr, args.stacks != nullptr);
    const size_t smem = tc_smem_bytes(bf16x3);
    cudaError_t e = prepare(fn, smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, kTcThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

// Resident CTAs per SM: kMinBlocks (the register file at 128 registers a
// thread; 128 tensor-memory columns each fill the SM's 512 at four); fewer if
// shared memory does not hold them.
int tc_max_ctas_per_sm(bool bf16x3, bool warm) {
    const TcKernel fn = tc_variant(bf16x3, warm, false);
    const size_t smem = tc_smem_bytes(bf16x3);
    if (prepare(fn, smem) != cudaSuccess) return 1;
    int dev = 0, per_sm = 0, reserved = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    const int by_smem = per_sm / (int)(smem + 1024 + reserved);  // + static shared memory
    const int n = by_smem < kMinBlocks ? by_smem : kMinBlocks;
    return n > 0 ? n : 1;
}

static_assert(kMinBlocks * (Plan<false>::BYTES + 2048) <= 228 * 1024 &&
                  kMinBlocks * (Plan<true>::BYTES + 2048) <= 228 * 1024,
              "kMinBlocks CTAs per SM");
static_assert(kMinBlocks * kTmemCols <= 512, "tensor memory of kMinBlocks CTAs");
static_assert(kTiles == 4 || kTiles == 8, "M = 64 or 128");
static_assert(Plan<false>::OFF_A1 % 1024 == 0 && Plan<true>::OFF_A1 % 1024 == 0, "alignment");

}  // namespace ncsb
