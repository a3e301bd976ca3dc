// ncs_warp_common.cuh -- device helpers of the warp-per-tile NCS solvers
// (ncs_warp.cu, ncs_spectral.cu): lane geometry, the 16x16 FFT pieces,
// warp reductions, the line-search log1p and tile gather helpers.
//
// Lane L of a warp holds rows P = L >> 2 and P + 8 at columns Qd + 4j
// (Qd = L & 3, j = 0..3) of its tile, packed as x[P][c] + i x[P+8][c].
#pragma once

#include "ncs_internal.cuh"

namespace ncsb {
namespace warp {


constexpr int kWarps = 4;
constexpr int kWarpCtaThreads = 32 * kWarps;
constexpr unsigned kFull = 0xffffffffu;
constexpr float kS2 = 0.70710678118654752f;  // sqrt(1/2)

// Per-warp shared memory (the history arrays follow it, sized by m).
struct WarpSmem {
    float2 fb[16][17];    // FFT transpose buffer
    float R[kMaxM][kMaxM];   // s_i'y_j by slot (upper triangle in age order is used)
    float YY[kMaxM][kMaxM];  // y_i'y_j by slot
    float rinv[kMaxM];       // 1 / s_i'y_i by slot
};

constexpr size_t kTableBytes = 256 * sizeof(float);

__host__ __device__ constexpr size_t warp_bytes(int m) {
    return ((sizeof(WarpSmem) + 15) / 16) * 16 + 2 * (size_t)m * 32 * 2 * sizeof(float4);
}

__device__ __forceinline__ int bitrev3(int i) {
    return ((i & 1) << 2) | (i & 2) | ((i & 4) >> 2);
}

// Packed FP32 pairs: sm_100's FADD2 / FMUL2 / FFMA2 issue both components as
// one instruction, each rounded as its scalar operation.  Complex values and
// the warp solvers' pixel pairs are such pairs.  Products with i swap the
// components, so the butterflies that take one (add_ib, sub_ib) stay scalar.
__device__ __forceinline__ float2 splat(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b exactly: the product b (-1) is exact and the sum rounds once
__device__ __forceinline__ float2 operator-(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// pixels 2j and 2j + 1 of a lane's 8 (rows P and P + 8 at column Qd + 4j) as a pair
__device__ __forceinline__ float2 pair(const float (&x)[8], int j) {
    return make_float2(x[2 * j], x[2 * j + 1]);
}
__device__ __forceinline__ void set_pair(float (&x)[8], int j, float2 z) {
    x[2 * j] = z.x;
    x[2 * j + 1] = z.y;
}
__device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }      // i a
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }     // -i a
__device__ __forceinline__ float2 add_ib(float2 a, float2 b) { return make_float2(a.x - b.y, a.y + b.x); }  // a + i b
__device__ __forceinline__ float2 sub_ib(float2 a, float2 b) { return make_float2(a.x + b.y, a.y - b.x); }  // a - i b
__device__ __forceinline__ float2 conjmul(float2 a, float2 w) {                            // a conj(w)
    return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y));
}
__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
    return make_float2(__shfl_xor_sync(kFull, v.x, m), __shfl_xor_sync(kFull, v.y, m));
}

// W16^p = exp(-2 pi i p / 16), p = 0..7
__device__ __forceinline__ float2 w16(int p) {
    const float c[8] = {1.0f, 0.92387953251128674f, kS2, 0.38268343236508978f,
                        0.0f, -0.38268343236508978f, -kS2, -0.92387953251128674f};
    const float s[8] = {0.0f, 0.38268343236508978f, kS2, 0.92387953251128674f,
                        1.0f, 0.92387953251128674f, kS2, 0.38268343236508978f};
    return make_float2(c[p], -s[p]);
}

// In-place 8-point DFT, decimation in frequency: natural order in, output
// position i holds frequency bitrev3(i).  Unnormalised.  The butterflies
// whose partner carries a factor -i are written as sub_ib / add_ib.
__device__ __forceinline__ void fft8_fwd(float2 (&e)[8]) {
    float2 a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        a[r] = e[r] + e[r + 4];
        b[r] = e[r] - e[r + 4];
    }
    // twiddles W8^1 and W8^3 (W8^2 = -i is taken by the butterflies below)
    const float2 t1 = make_float2(kS2 * (b[1].x + b[1].y), kS2 * (b[1].y - b[1].x));
    const float2 t3 = make_float2(kS2 * (b[3].y - b[3].x), -kS2 * (b[3].x + b[3].y));
    const float2 A0 = a[0] + a[2], A2 = a[0] - a[2], A1 = a[1] + a[3], A3 = a[1] - a[3];
    const float2 B0 = sub_ib(b[0], b[2]), B2 = add_ib(b[0], b[2]), B1 = t1 + t3, B3 = t1 - t3;
    e[0] = A0 + A1;
    e[1] = A0 - A1;
    e[2] = sub_ib(A2, A3);
    e[3] = add_ib(A2, A3);
    e[4] = B0 + B1;
    e[5] = B0 - B1;
    e[6] = sub_ib(B2, B3);
    e[7] = add_ib(B2, B3);
}

// Inverse of fft8_fwd up to the factor 8: bit-reversed in, natural out,
// conjugate twiddles (unnormalised inverse DFT).
__device__ __forceinline__ void fft8_inv(float2 (&e)[8]) {
    float2 a[8];
#pragma unroll
    for (int base = 0; base < 8; base += 2) {
        a[base] = e[base] + e[base + 1];
        a[base + 1] = e[base] - e[base + 1];
    }
    const float2 c0 = a[0] + a[2], c2 = a[0] - a[2], c1 = add_ib(a[1], a[3]), c3 = sub_ib(a[1], a[3]);
    const float2 c4 = a[4] + a[6], c6 = a[4] - a[6], c5 = add_ib(a[5], a[7]), c7 = sub_ib(a[5], a[7]);
    // conjugate twiddles W8^-1 and W8^-3 (W8^-2 = i is taken by the butterflies)
    const float2 t1 = make_float2(kS2 * (c5.x - c5.y), kS2 * (c5.x + c5.y));
    const float2 t3 = make_float2(-kS2 * (c7.x + c7.y), kS2 * (c7.x - c7.y));
    e[0] = c0 + c4;
    e[4] = c0 - c4;
    e[1] = c1 + t1;
    e[5] = c1 - t1;
    e[2] = add_ib(c2, c6);
    e[6] = sub_ib(c2, c6);
    e[3] = c3 + t3;
    e[7] = c3 - t3;
}

struct LaneGeo {
    int lane, P, Qd, KC, H, k0;
    float2 tw1, tw2, tw3;  // W16^(Qd*k1), k1 = 1..3
    float sA, sB, sH;      // butterfly signs of this lane
};

__device__ __forceinline__ LaneGeo lane_geo(int lane) {
    LaneGeo g;
    g.lane = lane;
    g.P = lane >> 2;
    g.Qd = lane & 3;
    g.KC = lane >> 1;
    g.H = lane & 1;
    g.k0 = 4 * ((g.Qd & 1) * 2 + (g.Qd >> 1));  // 4 * bitrev2(Qd)
    float sn, cs;
    sincospif((float)(g.Qd * 1) / 8.0f, &sn, &cs);
    g.tw1 = make_float2(cs, -sn);
    sincospif((float)(g.Qd * 2) / 8.0f, &sn, &cs);
    g.tw2 = make_float2(cs, -sn);
    sincospif((float)(g.Qd * 3) / 8.0f, &sn, &cs);
    g.tw3 = make_float2(cs, -sn);
    g.sA = g.Qd < 2 ? 1.0f : -1.0f;
    g.sB = (g.Qd & 1) ? -1.0f : 1.0f;
    g.sH = g.H ? -1.0f : 1.0f;
    return g;
}

// 128-bit shared-memory load that the compiler neither hoists out of a loop
// nor merges with an earlier one: a value re-read where it is used instead of
// held in a register across the solver's loop.
__device__ __forceinline__ float4 lds_v4_volatile(const void* p) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"((unsigned)__cvta_generic_to_shared(p)));
    return v;
}

// A history vector (s, y or Q s) of the warp solvers is stored as
// [half][lane] float4s, so that each 128-bit access of the warp covers 512
// consecutive bytes without bank conflicts (lane-major pairs of float4s
// would put two lanes on each bank).
__device__ __forceinline__ void load_hist(const float4* h, int lane, float (&x)[8]) {
    const float4 a = h[lane], b = h[32 + lane];
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}
__device__ __forceinline__ void store_hist(float4* h, int lane, const float (&x)[8]) {
    h[lane] = make_float4(x[0], x[1], x[2], x[3]);
    h[32 + lane] = make_float4(x[4], x[5], x[6], x[7]);
}

// The same as pixel pairs z[j] = (row P, row P + 8) at column Qd + 4j.
__device__ __forceinline__ void load_hist(const float4* h, int lane, float2 (&z)[4]) {
    const float4 a = h[lane], b = h[32 + lane];
    z[0] = make_float2(a.x, a.y);
    z[1] = make_float2(a.z, a.w);
    z[2] = make_float2(b.x, b.y);
    z[3] = make_float2(b.z, b.w);
}
__device__ __forceinline__ void store_hist(float4* h, int lane, const float2 (&z)[4]) {
    h[lane] = make_float4(z[0].x, z[0].y, z[1].x, z[1].y);
    h[32 + lane] = make_float4(z[2].x, z[2].y, z[3].x, z[3].y);
}

// The same, re-read at each use (not hoisted into registers across a loop).
__device__ __forceinline__ void load_hist_volatile(const float4* h, int lane, float2 (&z)[4]) {
    const float4 a = lds_v4_volatile(h + lane), b = lds_v4_volatile(h + 32 + lane);
    z[0] = make_float2(a.x, a.y);
    z[1] = make_float2(a.z, a.w);
    z[2] = make_float2(b.x, b.y);
    z[3] = make_float2(b.z, b.w);
}

// The pixel terms c = d + gamma and gamma of a lane's 8 pixels, kept in the
// warp's shared memory as [c low, c high, gamma low, gamma high][lane]
// float4s (each access is 32 consecutive 16-byte words) and re-read at
// every use.  Keeping them out of the loop-carried registers measured 2.6 %
// faster at the same occupancy: the solvers are issue-bound and the freed
// registers let the compiler schedule the transforms and the line search
// more tightly.  The loads are volatile so that they are not hoisted back
// out of the loop.
__device__ __forceinline__ void store_terms(float4* t, int lane, const float (&d)[8],
                                            const float (&gm)[8]) {
    t[lane] = make_float4(d[0] + gm[0], d[1] + gm[1], d[2] + gm[2], d[3] + gm[3]);
    t[32 + lane] = make_float4(d[4] + gm[4], d[5] + gm[5], d[6] + gm[6], d[7] + gm[7]);
    t[64 + lane] = make_float4(gm[0], gm[1], gm[2], gm[3]);
    t[96 + lane] = make_float4(gm[4], gm[5], gm[6], gm[7]);
}
__device__ __forceinline__ void load_terms(const float4* t, int lane, float (&c)[8],
                                           float (&gm)[8]) {
    const float4 c0 = lds_v4_volatile(t + lane), c1 = lds_v4_volatile(t + 32 + lane);
    const float4 g0 = lds_v4_volatile(t + 64 + lane), g1 = lds_v4_volatile(t + 96 + lane);
    c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
    c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
    gm[0] = g0.x; gm[1] = g0.y; gm[2] = g0.z; gm[3] = g0.w;
    gm[4] = g1.x; gm[5] = g1.y; gm[6] = g1.z; gm[7] = g1.w;
}

// The spectral solver's form of the pixel terms: -c and gamma as pixel pairs
// (the same layout), so that its packed updates take -c without negating.
__device__ __forceinline__ void store_terms_neg(float4* t, int lane, const float (&d)[8],
                                                const float (&gm)[8]) {
    t[lane] = make_float4(-(d[0] + gm[0]), -(d[1] + gm[1]), -(d[2] + gm[2]), -(d[3] + gm[3]));
    t[32 + lane] = make_float4(-(d[4] + gm[4]), -(d[5] + gm[5]), -(d[6] + gm[6]), -(d[7] + gm[7]));
    t[64 + lane] = make_float4(gm[0], gm[1], gm[2], gm[3]);
    t[96 + lane] = make_float4(gm[4], gm[5], gm[6], gm[7]);
}
__device__ __forceinline__ void load_terms_neg(const float4* t, int lane, float2 (&nc)[4],
                                               float2 (&gm)[4]) {
    const float4 c0 = lds_v4_volatile(t + lane), c1 = lds_v4_volatile(t + 32 + lane);
    const float4 g0 = lds_v4_volatile(t + 64 + lane), g1 = lds_v4_volatile(t + 96 + lane);
    nc[0] = make_float2(c0.x, c0.y);
    nc[1] = make_float2(c0.z, c0.w);
    nc[2] = make_float2(c1.x, c1.y);
    nc[3] = make_float2(c1.z, c1.w);
    gm[0] = make_float2(g0.x, g0.y);
    gm[1] = make_float2(g0.z, g0.w);
    gm[2] = make_float2(g1.x, g1.y);
    gm[3] = make_float2(g1.z, g1.w);
}

// The row-stage twiddles of the four lane classes Qd, for kernels that re-read
// them before each transform rather than keep six registers through the
// solve: v[Qd][0] = (tw1, tw2), v[Qd][1] = (tw3, unused).
struct TwiddleTable {
    float4 v[4][2];
};

// Threads 0..3 of the CTA fill the table (a __syncthreads must follow).
__device__ __forceinline__ void fill_twiddles(TwiddleTable& t, int tid) {
    if (tid < 4) {
        const LaneGeo g = lane_geo(tid);
        t.v[tid][0] = make_float4(g.tw1.x, g.tw1.y, g.tw2.x, g.tw2.y);
        t.v[tid][1] = make_float4(g.tw3.x, g.tw3.y, 0.0f, 0.0f);
    }
}

// A copy of the lane geometry with the twiddles freshly read from the table.
__device__ __forceinline__ LaneGeo with_twiddles(const LaneGeo& g, const TwiddleTable& t) {
    LaneGeo r = g;
    const float4 a = lds_v4_volatile(&t.v[g.Qd][0]), b = lds_v4_volatile(&t.v[g.Qd][1]);
    r.tw1 = make_float2(a.x, a.y);
    r.tw2 = make_float2(a.z, a.w);
    r.tw3 = make_float2(b.x, b.y);
    return r;
}

// Forward half of the 16x16 transform: lane (KC = L>>1, H = L&1) ends with
// the spectrum X[2 bitrev3(i) + H][KC] of its 8 pixels' tile in e[i]
// (unnormalised; with Halve = false, 2 X, for callers that fold the factor
// 1/2 of the row-pair separation into a later scaling).  Input: z[j] = rows
// P and P + 8 at column Qd + 4j, one complex row value.
template <bool Halve = true>
__device__ __forceinline__ void warp_fft_fwd(const float2 (&z)[4], float2 (&e)[8], WarpSmem& ws,
                                             const LaneGeo& L) {
    // rows: 4-point DFT over j in the lane, twiddle, 4-point DFT across lanes
    float2 V[4];
    {
        const float2 s02 = z[0] + z[2], d02 = z[0] - z[2], s13 = z[1] + z[3], d13 = z[1] - z[3];
        V[0] = s02 + s13;
        V[2] = cmul(s02 - s13, L.tw2);
        V[1] = cmul(sub_ib(d02, d13), L.tw1);
        V[3] = cmul(add_ib(d02, d13), L.tw3);
    }
    const bool q3 = L.Qd == 3;
    const float2 sA = splat(L.sA), sB = splat(L.sB);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 t = fma2(sA, V[k], shfl_xor2(V[k], 2));
        V[k] = q3 ? mul_mi(t) : t;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) V[k] = fma2(sB, V[k], shfl_xor2(V[k], 1));
    __syncwarp();  // previous users of the transpose buffer are done
#pragma unroll
    for (int k = 0; k < 4; ++k) ws.fb[L.P][L.k0 + k] = V[k];
    __syncwarp();

    // columns: lane (KC, H) separates the two packed rows of every row pair
    // from X[KC] and X[-KC], forms the even (H = 0) or odd (H = 1) half of the
    // 16-point column DFT and transforms it with an 8-point DFT.
    const int kneg = (16 - L.KC) & 15;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const float2 Z = ws.fb[p][L.KC], Zm = ws.fb[p][kneg];
        const float2 S = Z + Zm, D = Z - Zm;
        float2 ev = make_float2(fmaf(L.sH, S.y, S.x), fmaf(-L.sH, D.x, D.y));
        if (Halve) ev = ev * splat(0.5f);
        // odd half: twiddle W16^p (p = 0: 1; p = 4: -i, exact)
        if (p == 0) e[p] = ev;
        else if (p == 4) e[p] = L.H ? mul_mi(ev) : ev;
        else e[p] = L.H ? cmul(ev, w16(p)) : ev;
    }
    fft8_fwd(e);
}

// The same from 8 real pixels: x[2j] = row P, x[2j+1] = row P+8, column Qd + 4j.
template <bool Halve = true>
__device__ __forceinline__ void warp_fft_fwd(const float (&x)[8], float2 (&e)[8], WarpSmem& ws,
                                             const LaneGeo& L) {
    const float2 z[4] = {make_float2(x[0], x[1]), make_float2(x[2], x[3]),
                         make_float2(x[4], x[5]), make_float2(x[6], x[7])};
    warp_fft_fwd<Halve>(z, e, ws, L);
}

// Column stage of the inverse: from a spectrum in the layout warp_fft_fwd
// leaves, the even-frequency (H = 0) and twiddled odd-frequency (H = 1)
// halves of every column's inverse: fb[r][KC] = E_r and fb[r + 8][KC] = O_r,
// r = 0..7, so that row r of the row spectra is E_r + O_r and row r + 8 is
// E_r - O_r.  The reader combines them, which costs no shuffles.
__device__ __forceinline__ void warp_ifft_cols(float2 (&e)[8], WarpSmem& ws, const LaneGeo& L) {
    fft8_inv(e);
    // odd half: conjugate twiddle (r = 0: 1; r = 4: i, exact)
#pragma unroll
    for (int r = 1; r < 8; ++r)
        e[r] = L.H ? (r == 4 ? mul_i(e[r]) : conjmul(e[r], w16(r))) : e[r];
    __syncwarp();  // every lane has read the row spectra
#pragma unroll
    for (int r = 0; r < 8; ++r) ws.fb[r + 8 * L.H][L.KC] = e[r];
    __syncwarp();
}

// Row stage of the inverse: V[k] = one row's spectrum at frequencies k0 + k
// (this lane's four); z[j] = that row at column Qd + 4j (unnormalised).
__device__ __forceinline__ void warp_ifft_row(float2 (&V)[4], float2 (&z)[4], const LaneGeo& L) {
    const float2 sA = splat(L.sA), sB = splat(L.sB);
#pragma unroll
    for (int k = 0; k < 4; ++k) V[k] = fma2(sB, V[k], shfl_xor2(V[k], 1));
    // butterfly of lanes Qd and Qd ^ 2: lower = own + i^odd partner, upper =
    // partner - i^odd own.  The upper lane twiddles its own value before the
    // exchange, so each lane adds sA times its (twiddled) value to what it
    // receives: one select pair instead of three.
    const bool upper_odd = L.Qd == 3;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 y = upper_odd ? mul_i(V[k]) : V[k];
        V[k] = fma2(sA, y, shfl_xor2(y, 2));
    }
    V[1] = conjmul(V[1], L.tw1);
    V[2] = conjmul(V[2], L.tw2);
    V[3] = conjmul(V[3], L.tw3);
    const float2 s02 = V[0] + V[2], d02 = V[0] - V[2], s13 = V[1] + V[3], d13 = V[1] - V[3];
    z[0] = s02 + s13;
    z[2] = s02 - s13;
    z[1] = add_ib(d02, d13);
    z[3] = sub_ib(d02, d13);
}

// Inverse half: from a spectrum in the layout warp_fft_fwd leaves, the real
// tile back in this lane's pixel pairs (unnormalised inverse: x 256): z[j] =
// rows P and P + 8 at column Qd + 4j.  The two real rows share one complex
// row transform.
__device__ __forceinline__ void warp_fft_inv(float2 (&e)[8], float2 (&z)[4], WarpSmem& ws,
                                             const LaneGeo& L) {
    warp_ifft_cols(e, ws, L);
    float2 V[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        // rows P = E + O and P + 8 = E - O, packed as one complex row
        const float2 ev = ws.fb[L.P][L.k0 + k], od = ws.fb[L.P + 8][L.k0 + k];
        V[k] = add_ib(ev + od, ev - od);
    }
    warp_ifft_row(V, z, L);
}

// The same into 8 real pixels: y[2j] = row P, y[2j+1] = row P+8.
__device__ __forceinline__ void warp_fft_inv(float2 (&e)[8], float (&y)[8], WarpSmem& ws,
                                             const LaneGeo& L) {
    float2 z[4];
    warp_fft_inv(e, z, ws, L);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        y[2 * j] = z[j].x;
        y[2 * j + 1] = z[j].y;
    }
}

// y = Q x for the 8 pixels of this lane; mt = this lane's 8 values of
// M^2/256 in the column-pass layout.
__device__ __forceinline__ void warp_apply_q(const float (&x)[8], float (&y)[8], WarpSmem& ws,
                                             const float* mt, const LaneGeo& L, float* nc_part) {
    float2 e[8];
    warp_fft_fwd(x, e, ws, L);
    const float4 m0 = *reinterpret_cast<const float4*>(mt);
    const float4 m1 = *reinterpret_cast<const float4*>(mt + 4);
    const float mk[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
    if (nc_part) {
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) s = fmaf(fmaf(e[i].x, e[i].x, e[i].y * e[i].y), mk[i], s);
        *nc_part = s;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) e[i] = make_float2(e[i].x * mk[i], e[i].y * mk[i]);
    warp_fft_inv(e, y, ws, L);
}

// 1/x from the hardware reciprocal (PTX rcp.approx.ftz.f32: one MUFU
// operation, relative error about 2^-23, subnormals flushed).  The solvers
// only take reciprocals of values >= 1e-6 or of sums that are bounded away
// from 0, where it matches 1/x to FP32 precision.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// log(x) = log2(x) ln 2 from the hardware log2 (PTX lg2.approx.ftz.f32, one
// MUFU operation, absolute error about 2^-22 in log2), for x >= 1e-6.
__device__ __forceinline__ float log_fast(float x) {
    float l2;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"(x));
    return l2 * 0.69314718055994531f;  // ln 2
}

// log1p(x) for x > -1: 2 atanh(y), y = x / (2 + x), by the odd series
// 2y (1 + y^2/3 + ... + y^8/9) when |x| <= 1/2 (|y| <= 1/5, truncation
// < 1e-8 relative); otherwise log(1 + x) from the hardware log2, whose
// absolute error is small against |log(1 + x)| >= 0.4 there.
__device__ __forceinline__ float log1p_ls(float x) {
    const float y = x * rcp_fast(2.0f + x);
    const float y2 = y * y;
    // Horner on the doubled coefficients: exactly 2 s, so y (2 s) = (2 y) s
    float s = fmaf(y2, 2.0f / 9.0f, 2.0f / 7.0f);
    s = fmaf(y2, s, 2.0f / 5.0f);
    s = fmaf(y2, s, 2.0f / 3.0f);
    s = fmaf(y2, s, 2.0f);
    const float small = y * s;
    return fabsf(x) <= 0.5f ? small : log_fast(1.0f + x);
}

// log1p_ls of a pair: the arithmetic packed, the reciprocals, the log2s and
// the choice of branch per component.
__device__ __forceinline__ float2 log1p_ls(float2 x) {
    const float2 den = x + splat(2.0f);
    const float2 y = x * make_float2(rcp_fast(den.x), rcp_fast(den.y));
    const float2 y2 = y * y;
    float2 s = fma2(y2, splat(2.0f / 9.0f), splat(2.0f / 7.0f));
    s = fma2(y2, s, splat(2.0f / 5.0f));
    s = fma2(y2, s, splat(2.0f / 3.0f));
    s = fma2(y2, s, splat(2.0f));
    const float2 small = y * s;
    const float2 x1 = x + splat(1.0f);
    float2 l2;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2.x) : "f"(x1.x));
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2.y) : "f"(x1.y));
    const float2 big = l2 * splat(0.69314718055994531f);  // ln 2
    return make_float2(fabsf(x.x) <= 0.5f ? small.x : big.x, fabsf(x.y) <= 0.5f ? small.y : big.y);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Warp totals of four FP64 values: the first two levels exchange halves of
// the 4-slot vector, so lane L & 3 = j ends with total j after 6 double
// shuffles; 4 more broadcast them (20 for four plain sums).
__device__ __forceinline__ void warp_sum4_d(double& a, double& b, double& c, double& d, int lane) {
    const bool up2 = (lane & 2) != 0, up1 = (lane & 1) != 0;
    double v0 = (up2 ? c : a) + __shfl_xor_sync(kFull, up2 ? a : c, 2);
    double v1 = (up2 ? d : b) + __shfl_xor_sync(kFull, up2 ? b : d, 2);
    v0 = (up1 ? v1 : v0) + __shfl_xor_sync(kFull, up1 ? v0 : v1, 1);
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) v0 += __shfl_xor_sync(kFull, v0, o);
    a = __shfl_sync(kFull, v0, 0);
    b = __shfl_sync(kFull, v0, 1);
    c = __shfl_sync(kFull, v0, 2);
    d = __shfl_sync(kFull, v0, 3);
}

// Warp totals of three FP64 values: warp_sum4_d with slot 3 empty (6 double
// shuffles and 3 broadcasts; 15 for three plain sums).
__device__ __forceinline__ void warp_sum3_d(double& a, double& b, double& c, int lane) {
    const bool up2 = (lane & 2) != 0, up1 = (lane & 1) != 0;
    const double s0 = up2 ? a : c, s1 = up2 ? b : 0.0;
    double v0 = (up2 ? c : a) + __shfl_xor_sync(kFull, s0, 2);
    double v1 = (up2 ? 0.0 : b) + __shfl_xor_sync(kFull, s1, 2);
    v0 = (up1 ? v1 : v0) + __shfl_xor_sync(kFull, up1 ? v0 : v1, 1);
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) v0 += __shfl_xor_sync(kFull, v0, o);
    a = __shfl_sync(kFull, v0, 0);
    b = __shfl_sync(kFull, v0, 1);
    c = __shfl_sync(kFull, v0, 2);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ void load8(const float4* h, float (&x)[8]) {
    const float4 a = h[0], b = h[1];
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}

__device__ __forceinline__ void store8(float4* h, const float (&x)[8]) {
    h[0] = make_float4(x[0], x[1], x[2], x[3]);
    h[1] = make_float4(x[4], x[5], x[6], x[7]);
}

}  // namespace warp
}  // namespace ncsb
