// learned.cu — learned correction of a cheap MOG ensemble.
//
// No counterpart in the reference: its force is always the plain average
// over k grids (update.glsl:67-81).  Here a small network (12 -> 64 -> 64 -> 3,
// GELU) predicts, from statistics of a cheap ensemble (k = 32), the residual
// to an expensive one (k = 240).
//
// One fused kernel (learned_kernel) does, per particle:
//   gather    the k world-frame grid forces and cell masses it touches (L2),
//             accumulating the statistics of the features: the mean force,
//             a least-squares correction of it from the particle's offsets
//             to its cells' centres, the per-grid force spread, the mean
//             cell mass and two scalars (see gather_features);
//   inference the standardised features through the network on the tensor
//             cores (mma.sync m16n8k16 FP16, FP32 accumulate): a warp's 32
//             particles are two m16 tiles; the accumulator fragment of one
//             layer is, pair of n-tiles by pair, exactly the A fragment of
//             the next;
//   update    force = base + out_scale * y, then update.glsl:83-89.
// so nothing per particle but its position and velocity touches HBM.
// The same kernel also writes the features only (mog_features) or the
// corrected force only (mog_learned_forces).
//
//   training  FP32 fused forward + backward over a minibatch, one CTA per
//             128 samples, per-CTA partial gradients reduced in a fixed
//             order (deterministic), then Adam.
//
// Parameter vector layout (FP32, kParams floats):
//   W1[64][12] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
#include <algorithm>
#include <cstdint>
#include <cuda_fp16.h>

#include "mog_internal.h"

namespace mog {

constexpr int kIn = 12, kH = 64, kOut = 3;
constexpr int kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH,
              kW3 = kB2 + kH, kB3 = kW3 + kOut * kH, kParams = kB3 + kOut;
static_assert(kParams == 5187, "parameter count");

namespace {

// GELU, tanh form; gelu' for the backward pass.
__device__ __forceinline__ float gelu_f(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float u = 0.7978845608028654f * (x + 0.044715f * x2 * x);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * x2);
}
// ---------------------------------------------------------------------------
// FP16 weight fragments for mma.sync.m16n8k16 (B operand, "col" layout):
// for k-step ks and n-tile nt, lane l holds
//   b0 = {W[n][k], W[n][k+1]} with n = nt*8 + l/4, k = ks*16 + 2*(l%4)
//   b1 = the same at k + 8.
// Stored as uint2 [ks][nt][32] so a warp reads 256 contiguous bytes.
// Layer 1 carries its bias as input column 12 (the A tile holds a constant
// 1 there); layers 2 and 3 are packed at half their weights, because the
// activations they read are 2 gelu(x) (gelu2_h2).
constexpr int kFrag1 = 1 * 8, kFrag2 = 4 * 8, kFrag3 = 4 * 1;  // (k-steps x n-tiles)
constexpr int kFragTotal = (kFrag1 + kFrag2 + kFrag3) * 32;     // uint2 per model

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
    const __half2 v = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Twice the GELU (tanh form) of two FP32 pre-activations, evaluated in
// packed FP16: u = x (c1 + c2 x^2), t = tanh.approx.f16x2(u), x + x t =
// 2 gelu(x).  The result is the FP16 A operand of the next layer, whose
// weights are packed at half their value; the factors of 2 are exact.
__device__ __forceinline__ uint32_t gelu2_h2(float a, float b, uint32_t c1, uint32_t c2) {
    const uint32_t x = pack_h2(a, b);
    uint32_t x2, p, u, t, y;
    asm("mul.rn.f16x2 %0, %1, %1;" : "=r"(x2) : "r"(x));
    asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(p) : "r"(x2), "r"(c2), "r"(c1));
    asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(u) : "r"(x), "r"(p));
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(u));
    asm("fma.rn.f16x2 %0, %1, %2, %1;" : "=r"(y) : "r"(x), "r"(t));
    return y;
}

// (lo, hi) as FP16, values beyond the FP16 range clamped to its largest
// finite value (cvt .satfinite).
__device__ __forceinline__ uint32_t pack_h2_sat(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// sqrt (sqrt.approx.f32, relative error about 2^-23) for the features,
// which enter an FP16 network.
__device__ __forceinline__ float sqrt_feature(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__global__ void pack_fragments_kernel(const float* __restrict__ params, uint2* __restrict__ frags) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kFragTotal) return;
    const int lane = t & 31;
    int idx = t >> 5;  // fragment index over all layers
    const float* Wm;
    int in, out, ks, nt, ntiles;
    if (idx < kFrag1) {
        Wm = params + kW1; in = kIn; out = kH; ntiles = 8;
    } else if (idx < kFrag1 + kFrag2) {
        idx -= kFrag1; Wm = params + kW2; in = kH; out = kH; ntiles = 8;
    } else {
        idx -= kFrag1 + kFrag2; Wm = params + kW3; in = kH; out = kOut; ntiles = 1;
    }
    ks = idx / ntiles;
    nt = idx % ntiles;
    const int n = nt * 8 + (lane >> 2);
    const int k = ks * 16 + 2 * (lane & 3);
    const float scale = Wm == params + kW1 ? 1.0f : 0.5f;
    auto w = [&](int nn, int kk) {
        if (nn >= out) return 0.f;
        if (kk < in) return scale * Wm[nn * in + kk];
        return (Wm == params + kW1 && kk == in) ? params[kB1 + nn] : 0.f;  // layer 1's bias column
    };
    frags[t] = make_uint2(pack_h2(w(n, k), w(n, k + 1)), pack_h2(w(n, k + 8), w(n, k + 9)));
}

__device__ __forceinline__ void mma_f16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// Fused gather + features + inference + update.


// Statistics of one particle over the k grids.
//
// Each grid samples the force at the centre of the particle's cell, not at
// the particle, so the k per-grid forces F_i scatter around the force at
// the particle roughly linearly in the particle's offset from those cell
// centres, d_i (world frame).  A per-particle least-squares fit
// F_i ~ a + B d_i over the k grids gives an intercept a, the force
// extrapolated to the particle itself:
//     a = Fbar - C_Fd (C_dd + ridge)^-1 dbar
// with dbar, C_dd = cov(d, d) and C_Fd = cov(F, d) over the grids.
// The features (before standardisation with the model's mu / sigma) are
//   0-2  Fbar / s            plain ensemble mean (update.glsl order)
//   3-5  (a - Fbar) / s      regression correction from the in-cell offsets
//   6-8  std_i(F_i) / s      per-component spread of the per-grid forces
//   9    log1p(rho / rho_ref) mean mass of the particle's cells
//   10   |Fbar| / s
//   11   sqrt(tr C_dd) / h   spread of the in-cell offsets
// The cell masses come from the .w lane of the world-frame force grid
// (density_w_kernel puts them there).
struct Features {
    float f[kIn];
    float mx, my, mz;  // Fbar
    float ex, ey, ez;  // a - Fbar
};

__device__ __forceinline__ GridRows make_grid_rows_dev(const Ensemble& e, int i) {
    const FastXf x = e.fast[i];
    const float* R = e.rot12 + 12 * i;
    GridRows g;
    g.t01[0] = make_float2(x.row[0].x, x.row[1].x);
    g.t01[1] = make_float2(x.row[0].y, x.row[1].y);
    g.t01[2] = make_float2(x.row[0].z, x.row[1].z);
    g.t01[3] = make_float2(x.row[0].w, x.row[1].w);
    g.t2 = x.row[2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) g.m[3 * a + b] = R[4 * a + b] * e.voxel;
        g.o[a] = -0.5f * (g.m[3 * a] + g.m[3 * a + 1] + g.m[3 * a + 2]);
    }
    return g;
}

// Running sums of one particle over the grids.  Pairs of sums that take
// pairwise operands are float2, updated by one paired FP32 instruction
// (add/fma .f32x2: two IEEE operations, each rounded as the scalar one).
struct GatherAcc {
    float2 s01 = make_float2(0.f, 0.f);   // plain sum (x, y), update.glsl order
    float sz = 0.f;
    float2 q01 = make_float2(0.f, 0.f);   // sum F^2 (x, y)
    float qz = 0.f;
    float2 d01 = make_float2(0.f, 0.f);   // sum d (x, y)
    float dz = 0.f;
    float2 dd01 = make_float2(0.f, 0.f);  // sum (dx dx, dy dy)
    float dzz = 0.f, dxy = 0.f;
    float2 dz01 = make_float2(0.f, 0.f);  // sum (dx dz, dy dz)
    float2 fd_a = make_float2(0.f, 0.f);  // sum (Fx dx, Fy dy)
    float2 fd_b = make_float2(0.f, 0.f);  // sum (Fx dy, Fy dx)
    float2 fd_c = make_float2(0.f, 0.f);  // sum (Fx dz, Fy dz)
    float2 fd_d = make_float2(0.f, 0.f);  // sum (Fz dx, Fz dy)
    float fzdz = 0.f, rho = 0.f;
};

// Grid i's contribution.  IDX 0: FAST cells (LG = log2 g, or 0 for a
// run-time g); IDX 1: EXACT cells.  cc: the centred position's components
// each duplicated into a pair.  tx and ty come from paired FMAs in the
// order cell_fast uses, so the cell is the deposit's.  In FAST mode the
// floor that picks the cell also gives the offset: r = t + 1.5*2^23
// rounded down holds floor(t) in its low bits (the cell, as
// floor_mod_pow2) and r - 1.5*2^23 = floor(t) exactly, for |t| < 2^22.
template <int IDX, int LG>
__device__ __forceinline__ void gather_one(const GridRows& x, int i, const float4* __restrict__ W,
                                           const Ensemble& e, const IndexParams& ip, float cx,
                                           float cy, float cz, const float2 (&cc)[3],
                                           GatherAcc& a) {
    const int lg = LG > 0 ? LG : e.lg;
    const int G3 = 1 << (3 * lg);
    const uint32_t mask = (1u << lg) - 1u;
    constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
    const float2 txy = __ffma2_rn(x.t01[2], cc[2], __ffma2_rn(x.t01[1], cc[1],
                                                              __ffma2_rn(x.t01[0], cc[0], x.t01[3])));
    const float tz = __fmaf_rn(x.t2.z, cz, __fmaf_rn(x.t2.y, cy, __fmaf_rn(x.t2.x, cx, x.t2.w)));
    uint32_t c;
    float2 gxy;  // frac(t) for x, y
    float gz;
    if (IDX == 0) {
        const float2 rxy = __fadd2_rd(txy, make_float2(kMagic, kMagic));
        const float rz = __fadd_rd(tz, kMagic);
        c = (__float_as_uint(rxy.x) & mask) | ((__float_as_uint(rxy.y) & mask) << lg) |
            ((__float_as_uint(rz) & mask) << (2 * lg));
        // t - (r - 1.5*2^23): the inner difference is exact, the outer one a
        // single rounding, as t - floor(t)
        gxy = __ffma2_rn(__fadd2_rn(rxy, make_float2(-kMagic, -kMagic)), make_float2(-1.f, -1.f), txy);
        gz = tz - (rz - kMagic);
    } else {
        c = cell_exact(e.rot12 + 12 * i, e.off4 + 4 * i, cx, cy, cz, ip);
        gxy = make_float2(txy.x - floorf(txy.x), txy.y - floorf(txy.y));
        gz = tz - floorf(tz);
    }
    if (!in_bounds(e.flags, c, (uint64_t)G3)) c = 0;
    const float4 f = __ldg(W + (size_t)i * G3 + c);
    const float2 f01 = make_float2(f.x, f.y);
    a.s01 = __fadd2_rn(a.s01, f01);
    a.sz = __fadd_rn(a.sz, f.z);
    a.q01 = __ffma2_rn(f01, f01, a.q01);
    a.qz = __fmaf_rn(f.z, f.z, a.qz);
    // world-frame offset from the cell centre: (h M) frac(t) + o
    const float wx = __fmaf_rn(x.m[2], gz, __fmaf_rn(x.m[1], gxy.y, __fmaf_rn(x.m[0], gxy.x, x.o[0])));
    const float wy = __fmaf_rn(x.m[5], gz, __fmaf_rn(x.m[4], gxy.y, __fmaf_rn(x.m[3], gxy.x, x.o[1])));
    const float wz = __fmaf_rn(x.m[8], gz, __fmaf_rn(x.m[7], gxy.y, __fmaf_rn(x.m[6], gxy.x, x.o[2])));
    const float2 w01 = make_float2(wx, wy), wzz = make_float2(wz, wz);
    a.d01 = __fadd2_rn(a.d01, w01);
    a.dz = __fadd_rn(a.dz, wz);
    a.dd01 = __ffma2_rn(w01, w01, a.dd01);
    a.dzz = __fmaf_rn(wz, wz, a.dzz);
    a.dxy = __fmaf_rn(wx, wy, a.dxy);
    a.dz01 = __ffma2_rn(w01, wzz, a.dz01);
    a.fd_a = __ffma2_rn(f01, w01, a.fd_a);
    a.fd_b = __ffma2_rn(f01, make_float2(wy, wx), a.fd_b);
    a.fd_c = __ffma2_rn(f01, wzz, a.fd_c);
    a.fd_d = __ffma2_rn(make_float2(f.z, f.z), w01, a.fd_d);
    a.fzdz = __fmaf_rn(f.z, wz, a.fzdz);
    a.rho = __fadd_rn(a.rho, f.w);
}

// Features from the sums over k grids of voxel size h.  EXACT_MEAN: the
// mean force Fbar divides by k with IEEE division, bit-identical to the plain
// gather's average (mog_features); otherwise it multiplies by 1/k (the same
// value when k is a power of two).  Square roots, the logarithm and 1/det
// use the approximate forms: the features enter an FP16 network.
template <bool EXACT_MEAN>
__device__ __forceinline__ void finish_features(const GatherAcc& a, int k, float h, float inv_fs,
                                                float rho_ref, Features& out) {
    const float sx = a.s01.x, sy = a.s01.y, sz = a.sz, qx = a.q01.x, qy = a.q01.y, qz = a.qz;
    const float dx = a.d01.x, dy = a.d01.y, dz = a.dz, dxx = a.dd01.x, dxy = a.dxy,
                dxz = a.dz01.x, dyy = a.dd01.y, dyz = a.dz01.y, dzz = a.dzz;
    const float fxdx = a.fd_a.x, fxdy = a.fd_b.x, fxdz = a.fd_c.x, fydx = a.fd_b.y,
                fydy = a.fd_a.y, fydz = a.fd_c.y, fzdx = a.fd_d.x, fzdy = a.fd_d.y, fzdz = a.fzdz,
                rho = a.rho;
    const float kf = (float)k, ik = 1.0f / kf;
    const float mx = EXACT_MEAN ? __fdiv_rn(sx, kf) : sx * ik;
    const float my = EXACT_MEAN ? __fdiv_rn(sy, kf) : sy * ik;
    const float mz = EXACT_MEAN ? __fdiv_rn(sz, kf) : sz * ik;
    const float ax_ = dx * ik, ay_ = dy * ik, az_ = dz * ik;  // dbar
    const float ridge = 1e-3f * h * h;
    const float cxx = dxx * ik - ax_ * ax_ + ridge, cxy = dxy * ik - ax_ * ay_,
                cxz = dxz * ik - ax_ * az_, cyy = dyy * ik - ay_ * ay_ + ridge,
                cyz = dyz * ik - ay_ * az_, czz = dzz * ik - az_ * az_ + ridge;
    // solve C_dd w = dbar (symmetric 3x3, adjugate)
    const float A00 = cyy * czz - cyz * cyz, A01 = cxz * cyz - cxy * czz, A02 = cxy * cyz - cxz * cyy;
    const float A11 = cxx * czz - cxz * cxz, A12 = cxy * cxz - cxx * cyz, A22 = cxx * cyy - cxy * cxy;
    const float det = cxx * A00 + cxy * A01 + cxz * A02;
    float wx = 0.f, wy = 0.f, wz = 0.f;
    if (det > 0.f) {
        const float id = __frcp_rn(det);
        wx = (A00 * ax_ + A01 * ay_ + A02 * az_) * id;
        wy = (A01 * ax_ + A11 * ay_ + A12 * az_) * id;
        wz = (A02 * ax_ + A12 * ay_ + A22 * az_) * id;
    }
    // correction = -C_Fd w,  C_Fd = sum(F d^T)/k - Fbar dbar^T
    out.ex = -((fxdx * ik - mx * ax_) * wx + (fxdy * ik - mx * ay_) * wy + (fxdz * ik - mx * az_) * wz);
    out.ey = -((fydx * ik - my * ax_) * wx + (fydy * ik - my * ay_) * wy + (fydz * ik - my * az_) * wz);
    out.ez = -((fzdx * ik - mz * ax_) * wx + (fzdy * ik - mz * ay_) * wy + (fzdz * ik - mz * az_) * wz);
    out.mx = mx;
    out.my = my;
    out.mz = mz;
    out.f[0] = mx * inv_fs;
    out.f[1] = my * inv_fs;
    out.f[2] = mz * inv_fs;
    out.f[3] = out.ex * inv_fs;
    out.f[4] = out.ey * inv_fs;
    out.f[5] = out.ez * inv_fs;
    out.f[6] = sqrt_feature(fmaxf(qx * ik - mx * mx, 0.f)) * inv_fs;
    out.f[7] = sqrt_feature(fmaxf(qy * ik - my * my, 0.f)) * inv_fs;
    out.f[8] = sqrt_feature(fmaxf(qz * ik - mz * mz, 0.f)) * inv_fs;
    out.f[9] = __logf(1.0f + rho * ik / rho_ref);
    out.f[10] = sqrt_feature(mx * mx + my * my + mz * mz) * inv_fs;
    out.f[11] = sqrt_feature(fmaxf(cxx + cyy + czz - 3.f * ridge, 0.f)) * (1.0f / h);
}

// The network on one m16 tile of a warp: A fragment (a0..a3) of the
// standardised features in, y fragment of the 8-wide output tile out
// (outputs 0..2 live).  sf: weight fragments, sb: b1 | b2 | b3 (padded to 8).
__device__ __forceinline__ void mlp_tile(const uint2* __restrict__ sf, const float* __restrict__ sb,
                                         uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         int lane, float (&y)[4]) {
    const int tg = lane & 3;
    const uint32_t c1 = pack_h2(0.7978845608028654f, 0.7978845608028654f);
    const uint32_t c2 = pack_h2(0.7978845608028654f * 0.044715f, 0.7978845608028654f * 0.044715f);
    float h[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        // layer 1's bias comes in through the constant input column
        h[nt][0] = h[nt][1] = h[nt][2] = h[nt][3] = 0.f;
        const uint2 w = sf[(0 * 8 + nt) * 32 + lane];
        mma_f16(h[nt], a0, a1, a2, a3, w.x, w.y);
    }
    uint32_t A[4][4];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        A[ks][0] = gelu2_h2(h[2 * ks][0], h[2 * ks][1], c1, c2);
        A[ks][1] = gelu2_h2(h[2 * ks][2], h[2 * ks][3], c1, c2);
        A[ks][2] = gelu2_h2(h[2 * ks + 1][0], h[2 * ks + 1][1], c1, c2);
        A[ks][3] = gelu2_h2(h[2 * ks + 1][2], h[2 * ks + 1][3], c1, c2);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float b0 = sb[kH + nt * 8 + 2 * tg], b1 = sb[kH + nt * 8 + 2 * tg + 1];
        h[nt][0] = b0; h[nt][1] = b1; h[nt][2] = b0; h[nt][3] = b1;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const uint2 w = sf[(kFrag1 + ks * 8 + nt) * 32 + lane];
            mma_f16(h[nt], A[ks][0], A[ks][1], A[ks][2], A[ks][3], w.x, w.y);
        }
    }
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        A[ks][0] = gelu2_h2(h[2 * ks][0], h[2 * ks][1], c1, c2);
        A[ks][1] = gelu2_h2(h[2 * ks][2], h[2 * ks][3], c1, c2);
        A[ks][2] = gelu2_h2(h[2 * ks + 1][0], h[2 * ks + 1][1], c1, c2);
        A[ks][3] = gelu2_h2(h[2 * ks + 1][2], h[2 * ks + 1][3], c1, c2);
    }
    y[0] = sb[2 * kH + 2 * tg];
    y[1] = sb[2 * kH + 2 * tg + 1];
    y[2] = y[0];
    y[3] = y[1];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        const uint2 w = sf[(kFrag1 + kFrag2 + ks) * 32 + lane];
        mma_f16(y, A[ks][0], A[ks][1], A[ks][2], A[ks][3], w.x, w.y);
    }
}

constexpr int kLT = 256;       // threads of learned_kernel
constexpr int kLW = kLT / 32;  // warps
constexpr int kARow = 12;      // u32 per A-tile row (8 used; 12 keeps the fragment loads conflict-free)
constexpr size_t kLearnedFixedSmem = sizeof(uint2) * kFragTotal + sizeof(float) * (2 * kH + 8) +
                                     sizeof(uint32_t) * kLW * 32 * kARow + sizeof(float4) * kLW * 32;
static_assert(kLearnedFixedSmem % 16 == 0, "GridRows must stay 16-byte aligned");

// OUT 0: one damped leapfrog step with the corrected force (pos, vel);
// OUT 1: the corrected force into out4;  OUT 2: the features (out4 = Fbar,
// feat = 16 floats: 0-11 standardised, 12-14 a - Fbar, 15 zero), no network.
// One thread per particle; a persistent grid walks blocks of kLT particles.
// The grid rows of a K-grid ensemble as a launch parameter: read through
// the constant cache with compile-time offsets once the grid loop is
// unrolled, so the gather issues no shared-memory loads for them.
template <int K>
struct GridTable {
    GridRows r[K > 0 ? K : 1];
};

// K > 0: k == K and the rows come from `tab`; K == 0: any k, rows staged in
// shared memory.
template <int IDX, int LG, int OUT, int K, int MINB = 2>
__global__ void __launch_bounds__(kLT, MINB) learned_kernel(
    float4* __restrict__ pos, float4* __restrict__ vel, int64_t n, const float4* __restrict__ W,
    Ensemble e, ModelNorm norm, const uint2* __restrict__ frags, const float* __restrict__ params,
    float dt, float damp, float4* __restrict__ out4, float* __restrict__ feat_out,
    float* __restrict__ spread_part, const __grid_constant__ GridTable<K> tab) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint2* sf = reinterpret_cast<uint2*>(smem_raw);
    float* sb = reinterpret_cast<float*>(sf + kFragTotal);
    uint32_t* sA = reinterpret_cast<uint32_t*>(sb + 2 * kH + 8);
    float4* sY = reinterpret_cast<float4*>(sA + kLW * 32 * kARow);
    GridRows* xf = reinterpret_cast<GridRows*>(smem_raw + kLearnedFixedSmem);
    if constexpr (K == 0) {
        for (int i = threadIdx.x; i < e.k; i += kLT) xf[i] = make_grid_rows_dev(e, i);
    }
    if (OUT != 2) {
        for (int i = threadIdx.x; i < kFragTotal; i += kLT) sf[i] = frags[i];
        for (int i = threadIdx.x; i < kH; i += kLT) {
            sb[i] = params[kB1 + i];
            sb[kH + i] = params[kB2 + i];
        }
        if (threadIdx.x < 8) sb[2 * kH + threadIdx.x] = threadIdx.x < kOut ? params[kB3 + threadIdx.x] : 0.f;
    }
    __syncthreads();
    // Launched as a programmatic dependent of the solve (launch_learned), this
    // grid may start while the solve still runs: the prologue above reads
    // only the model and the transforms; the force grid, written by the
    // solve, is read after this wait (a no-op without the dependency).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const IndexParams ip = e.index_params();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tg = lane & 3;
    uint32_t* A = sA + warp * 32 * kARow;
    float4* Y = sY + warp * 32;
    const float inv_fs = 1.0f / norm.force_scale;
    unsigned bad = 0;
    float spread = 0.f;  // sum over this thread's particles of mean(features 6-8)
    float fmag = 0.f;    // sum over this thread's particles of feature 10
    for (int64_t base = (int64_t)blockIdx.x * kLT; base < n; base += (int64_t)gridDim.x * kLT) {
        if (base + warp * 32 >= n) continue;  // whole warp past the end (warp-uniform)
        const int64_t p = base + threadIdx.x;
        const bool live = p < n;
        const float4 P = live ? pos[p] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float cx = __fsub_rn(P.x, ip.half_l), cy = __fsub_rn(P.y, ip.half_l),
                    cz = __fsub_rn(P.z, ip.half_l);
        GatherAcc acc;
        const float2 cc[3] = {make_float2(cx, cx), make_float2(cy, cy), make_float2(cz, cz)};
        if constexpr (K > 0) {
#pragma unroll
            for (int i = 0; i < K; ++i) gather_one<IDX, LG>(tab.r[i], i, W, e, ip, cx, cy, cz, cc, acc);
        } else {
#pragma unroll 4
            for (int i = 0; i < e.k; ++i) gather_one<IDX, LG>(xf[i], i, W, e, ip, cx, cy, cz, cc, acc);
        }
        Features F;
        finish_features<OUT == 2>(acc, e.k, e.voxel, inv_fs, norm.rho_ref, F);
        float z[kIn];
#pragma unroll
        for (int j = 0; j < kIn; ++j) z[j] = (F.f[j] - norm.mu[j]) * norm.inv_sigma[j];
        if constexpr (OUT == 2) {
            if (live) {
                out4[p] = make_float4(F.mx, F.my, F.mz, 0.f);
                float4* o = reinterpret_cast<float4*>(feat_out + (size_t)p * 16);
                o[0] = make_float4(z[0], z[1], z[2], z[3]);
                o[1] = make_float4(z[4], z[5], z[6], z[7]);
                o[2] = make_float4(z[8], z[9], z[10], z[11]);
                o[3] = make_float4(F.ex, F.ey, F.ez, 0.f);
            }
        } else {
            // this particle's row of the warp's A tile (FP16 pairs, clamped to the
            // FP16 range; column 12 the constant 1 of layer 1's bias, 13-15 zero)
            uint4* row = reinterpret_cast<uint4*>(A + lane * kARow);
            row[0] = make_uint4(pack_h2_sat(z[0], z[1]), pack_h2_sat(z[2], z[3]),
                                pack_h2_sat(z[4], z[5]), pack_h2_sat(z[6], z[7]));
            row[1] = make_uint4(pack_h2_sat(z[8], z[9]), pack_h2_sat(z[10], z[11]), 0x3c00u, 0u);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const uint32_t* Am = A + 16 * m * kARow;
                float y[4];
                mlp_tile(sf, sb, Am[g * kARow + tg], Am[(g + 8) * kARow + tg], Am[g * kARow + tg + 4],
                         Am[(g + 8) * kARow + tg + 4], lane, y);
                // y: rows g and g+8, outputs 2tg and 2tg+1
                if (tg == 0) {
                    Y[16 * m + g].x = y[0];
                    Y[16 * m + g].y = y[1];
                    Y[16 * m + g + 8].x = y[2];
                    Y[16 * m + g + 8].y = y[3];
                } else if (tg == 1) {
                    Y[16 * m + g].z = y[0];
                    Y[16 * m + g + 8].z = y[2];
                }
            }
            __syncwarp();
            const float4 yv = Y[lane];
            __syncwarp();  // the next block of particles reuses A and Y
            if (!live) continue;
            spread += (F.f[6] + F.f[7] + F.f[8]) * (1.0f / 3.0f);
            fmag += F.f[10];
            float bx = F.mx, by = F.my, bz = F.mz;
            if (norm.base_mode != 0.f) {
                bx += F.ex;
                by += F.ey;
                bz += F.ez;
            }
            const float ax = bx + norm.out_scale * yv.x, ay = by + norm.out_scale * yv.y,
                        az = bz + norm.out_scale * yv.z;
            if (OUT == 1) {
                out4[p] = make_float4(ax, ay, az, 0.f);
                continue;
            }
            // update.glsl:83-89 with the corrected force
            const float4 V = vel[p];
            const float vx = __fmul_rn(__fsub_rn(V.x, __fmul_rn(ax, dt)), damp);
            const float vy = __fmul_rn(__fsub_rn(V.y, __fmul_rn(ay, dt)), damp);
            const float vz = __fmul_rn(__fsub_rn(V.z, __fmul_rn(az, dt)), damp);
            const float px = glsl_mod(__fadd_rn(P.x, __fmul_rn(vx, dt)), e.world);
            const float py = glsl_mod(__fadd_rn(P.y, __fmul_rn(vy, dt)), e.world);
            const float pz = glsl_mod(__fadd_rn(P.z, __fmul_rn(vz, dt)), e.world);
            if (!(isfinite(px) && isfinite(py) && isfinite(pz))) bad |= 1u;  // MOG_FLAG_NONFINITE
            pos[p] = make_float4(px, py, pz, P.w);
            vel[p] = make_float4(vx, vy, vz, 0.f);
        }
    }
    if (bad) raise_flags(e.flags, bad);
    if (spread_part) {
        // per-CTA sums in a fixed order (warp shuffles, then thread 0)
        __shared__ float red[2][kLW];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            spread += __shfl_xor_sync(kFull, spread, o);
            fmag += __shfl_xor_sync(kFull, fmag, o);
        }
        if (lane == 0) {
            red[0][warp] = spread;
            red[1][warp] = fmag;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float a = 0.f, b = 0.f;
#pragma unroll
            for (int w = 0; w < kLW; ++w) {
                a += red[0][w];
                b += red[1][w];
            }
            spread_part[2 * blockIdx.x] = a;
            spread_part[2 * blockIdx.x + 1] = b;
        }
    }
}

// Cell masses into the .w lane of the world-frame force grid (which the
// world-frame solve leaves 0), clearing the mass grid for the next deposit.
// Also checks the deposit's fixed-point total for overflow and clears it,
// as the solve does when it clears the mass grid itself.
template <typename Acc>
__global__ void density_w_kernel(Acc* __restrict__ mass, float4* __restrict__ W, int64_t cells,
                                 float inv_scale, double* mass_total, unsigned* flags) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && mass_total) {
        if (*mass_total >= 18446744073709551616.0) atomicOr(flags, 2u);  // MOG_FLAG_OVERFLOW
        *mass_total = 0.0;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
         i += (int64_t)gridDim.x * blockDim.x) {
        reinterpret_cast<float*>(W + i)[3] = mass_value(mass[i], inv_scale);
        mass[i] = 0;
    }
}
// ---------------------------------------------------------------------------
// FP32 training: forward + backward for 128 samples per CTA.
constexpr int kTB = 128;   // samples per CTA
constexpr int kLd = kH + 1;  // padded row of an activation matrix

__global__ void __launch_bounds__(kTB) mlp_train_kernel(const float* __restrict__ feat,
                                                        const float* __restrict__ target,
                                                        const int* __restrict__ idx, int batch,
                                                        const float* __restrict__ params,
                                                        float* __restrict__ partial,
                                                        float* __restrict__ loss_partial) {
    extern __shared__ float sm[];
    float* w = sm;                         // kParams
    float* x = w + kParams;                // kTB x 12
    float* a1 = x + kTB * kIn;             // kTB x kLd (pre-activation, then its gradient)
    float* h1 = a1 + kTB * kLd;
    float* a2 = h1 + kTB * kLd;
    float* h2 = a2 + kTB * kLd;
    float* dy = h2 + kTB * kLd;            // kTB x 4 (3 used)
    const int t = threadIdx.x;
    for (int i = t; i < kParams; i += kTB) w[i] = params[i];
    const int s0 = blockIdx.x * kTB;
    const int s = s0 + t;
    const bool valid = s < batch;
    const int row = valid ? idx[s] : 0;
    for (int j = 0; j < kIn; ++j) x[t * kIn + j] = valid ? feat[(size_t)row * 16 + j] : 0.f;
    __syncthreads();
    // forward: one sample per thread, weights broadcast from shared memory
    for (int j = 0; j < kH; ++j) {
        float a = w[kB1 + j];
        for (int i = 0; i < kIn; ++i) a += w[kW1 + j * kIn + i] * x[t * kIn + i];
        a1[t * kLd + j] = a;
        h1[t * kLd + j] = gelu_f(a);
    }
    for (int j = 0; j < kH; ++j) {
        float a = w[kB2 + j];
        for (int i = 0; i < kH; ++i) a += w[kW2 + j * kH + i] * h1[t * kLd + i];
        a2[t * kLd + j] = a;
        h2[t * kLd + j] = gelu_f(a);
    }
    float loss = 0.f;
    for (int c = 0; c < kOut; ++c) {
        float y = w[kB3 + c];
        for (int i = 0; i < kH; ++i) y += w[kW3 + c * kH + i] * h2[t * kLd + i];
        const float d = valid ? y - target[(size_t)row * 4 + c] : 0.f;
        loss += d * d;
        dy[t * 4 + c] = valid ? 2.0f * d / (float)batch : 0.f;
    }
    // backward, per sample: gradients w.r.t. pre-activations, in place of a2 / a1
    for (int i = 0; i < kH; ++i) {
        float d = 0.f;
        for (int c = 0; c < kOut; ++c) d += w[kW3 + c * kH + i] * dy[t * 4 + c];
        a2[t * kLd + i] = d * gelu_grad(a2[t * kLd + i]);
    }
    for (int i = 0; i < kH; ++i) {
        float d = 0.f;
        for (int j = 0; j < kH; ++j) d += w[kW2 + j * kH + i] * a2[t * kLd + j];
        a1[t * kLd + i] = d * gelu_grad(a1[t * kLd + i]);
    }
    __syncthreads();
    // parameter gradients: each thread owns parameters, sums over samples in order
    for (int q = t; q < kParams; q += kTB) {
        float acc = 0.f;
        if (q < kB1) {
            const int j = q / kIn, i = q % kIn;
            for (int r = 0; r < kTB; ++r) acc += a1[r * kLd + j] * x[r * kIn + i];
        } else if (q < kW2) {
            const int j = q - kB1;
            for (int r = 0; r < kTB; ++r) acc += a1[r * kLd + j];
        } else if (q < kB2) {
            const int j = (q - kW2) / kH, i = (q - kW2) % kH;
            for (int r = 0; r < kTB; ++r) acc += a2[r * kLd + j] * h1[r * kLd + i];
        } else if (q < kW3) {
            const int j = q - kB2;
            for (int r = 0; r < kTB; ++r) acc += a2[r * kLd + j];
        } else if (q < kB3) {
            const int c = (q - kW3) / kH, i = (q - kW3) % kH;
            for (int r = 0; r < kTB; ++r) acc += dy[r * 4 + c] * h2[r * kLd + i];
        } else {
            const int c = q - kB3;
            for (int r = 0; r < kTB; ++r) acc += dy[r * 4 + c];
        }
        partial[(size_t)blockIdx.x * kParams + q] = acc;
    }
    // loss (sum of squares) per CTA, reduced in fixed order
    __shared__ float red[kTB];
    red[t] = loss;
    __syncthreads();
    if (t == 0) {
        float l = 0.f;
        for (int r = 0; r < kTB; ++r) l += red[r];
        loss_partial[blockIdx.x] = l;
    }
}

__global__ void reduce_grad_kernel(const float* __restrict__ partial, int ctas,
                                   float* __restrict__ grad) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams) return;
    float s = 0.f;
    for (int c = 0; c < ctas; ++c) s += partial[(size_t)c * kParams + q];
    grad[q] = s;
}

__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grad,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams) return;
    const float gq = grad[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    params[q] -= lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
}

}  // namespace

int mlp_param_count() { return kParams; }
size_t mlp_fragment_bytes() { return sizeof(uint2) * kFragTotal; }
size_t mlp_train_smem() {
    return sizeof(float) * ((size_t)kParams + kTB * kIn + 4 * kTB * kLd + kTB * 4);
}

cudaError_t launch_density_w(const Ensemble& e, void* mass, float4* W, cudaStream_t s) {
    const int64_t cells = e.cells();  // k * g^3
    const unsigned blocks = (unsigned)std::min<int64_t>((cells + 255) / 256, (int64_t)num_sms() * 8);
    if (e.mass_mode == 0)
        density_w_kernel<<<blocks, 256, 0, s>>>(static_cast<unsigned long long*>(mass), W, cells,
                                                e.inv_scale, e.mass_total, e.flags);
    else
        density_w_kernel<<<blocks, 256, 0, s>>>(static_cast<unsigned*>(mass), W, cells, e.inv_scale,
                                                nullptr, e.flags);
    return cudaGetLastError();
}

GridRows make_grid_rows(const FastXf& fast, const float* R, float voxel) {
    GridRows g;
    g.t01[0] = make_float2(fast.row[0].x, fast.row[1].x);
    g.t01[1] = make_float2(fast.row[0].y, fast.row[1].y);
    g.t01[2] = make_float2(fast.row[0].z, fast.row[1].z);
    g.t01[3] = make_float2(fast.row[0].w, fast.row[1].w);
    g.t2 = fast.row[2];
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) g.m[3 * a + b] = R[4 * a + b] * voxel;
        g.o[a] = -0.5f * (g.m[3 * a] + g.m[3 * a + 1] + g.m[3 * a + 2]);
    }
    return g;
}

namespace {
template <int IDX, int LG, int OUT, int K>
cudaError_t launch_learned_t(const Ensemble& e, const GridRows* rows, float4* pos, float4* vel,
                             int64_t n, const float4* W, const ModelNorm& norm, const void* frags,
                             const float* params, float dt, float damp, LearnedOut& out,
                             cudaStream_t s, int ctas_per_sm) {
    // three CTAs per SM (80 registers, some spilled) on request, where the
    // rows are launch parameters
    auto kern = (K > 0 && ctas_per_sm == 3) ? learned_kernel<IDX, LG, OUT, K, 3>
                                            : learned_kernel<IDX, LG, OUT, K, 2>;
    GridTable<K> tab{};
    if (K > 0)
        for (int i = 0; i < K; ++i) tab.r[i] = rows[i];
    const size_t smem = kLearnedFixedSmem + (K > 0 ? 0 : sizeof(GridRows) * (size_t)e.k);
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLT, smem);
    if (err != cudaSuccess) return err;
    int64_t blocks = std::min<int64_t>((n + kLT - 1) / kLT, (int64_t)num_sms() * std::max(per_sm, 1));
    if (out.spread && blocks > out.spread_cap) blocks = out.spread_cap;
    out.blocks = (int)blocks;
    // programmatic dependent launch: the CTAs may be scheduled on the SMs the
    // solve leaves idle (at k = 32 it runs 16 CTAs) and load the model while
    // it finishes; the kernel waits for the solve before reading its grid
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(kLT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, pos, vel, n, W, e, norm, static_cast<const uint2*>(frags),
                              params, dt, damp, out.out4, out.feat, out.spread, tab);
}

template <int IDX, int LG, int K>
cudaError_t launch_learned_i(int out_mode, const Ensemble& e, const GridRows* rows, float4* pos,
                             float4* vel, int64_t n, const float4* W, const ModelNorm& norm,
                             const void* frags, const float* params, float dt, float damp,
                             LearnedOut& out, cudaStream_t s, int cps) {
    switch (out_mode) {
        case 0: return launch_learned_t<IDX, LG, 0, K>(e, rows, pos, vel, n, W, norm, frags, params, dt, damp, out, s, cps);
        case 1: return launch_learned_t<IDX, LG, 1, K>(e, rows, pos, vel, n, W, norm, frags, params, dt, damp, out, s, cps);
        default: return launch_learned_t<IDX, LG, 2, K>(e, rows, pos, vel, n, W, norm, frags, params, dt, damp, out, s, cps);
    }
}
}  // namespace

cudaError_t launch_learned(int out_mode, const Ensemble& e, const GridRows* rows, float4* pos,
                           float4* vel, int64_t n, const float4* W, const ModelNorm& norm,
                           const void* frags, const float* params, float dt, float damp,
                           LearnedOut& out, cudaStream_t s, int ctas_per_sm) {
    out.blocks = 0;
    if (n <= 0) return cudaSuccess;
#define MOG_LEARNED(IDX, LG, K) \
    return launch_learned_i<IDX, LG, K>(out_mode, e, rows, pos, vel, n, W, norm, frags, params, dt, damp, out, s, \
                                        ctas_per_sm)
    // the k = 32, g = 16 FAST ensemble (the cheap ensemble the models are
    // trained for) gets its rows as launch parameters and an unrolled loop
    if (e.index_mode == 0 && e.lg == 4 && e.k == 32 && rows) MOG_LEARNED(0, 4, 32);
    if (e.index_mode != 0) MOG_LEARNED(1, 0, 0);
    if (e.lg == 4) MOG_LEARNED(0, 4, 0);
    if (e.lg == 3) MOG_LEARNED(0, 3, 0);
    MOG_LEARNED(0, 0, 0);
#undef MOG_LEARNED
}

cudaError_t launch_pack_fragments(const float* params, void* frags, cudaStream_t s) {
    pack_fragments_kernel<<<(kFragTotal + 255) / 256, 256, 0, s>>>(params, static_cast<uint2*>(frags));
    return cudaGetLastError();
}

cudaError_t launch_mlp_train_step(const float* feat, const float* target, const int* idx,
                                  int batch, float* params, float* partial, float* loss_partial,
                                  float* grad, float* m, float* v, float lr, int t,
                                  cudaStream_t s) {
    const int ctas = (batch + kTB - 1) / kTB;
    const size_t smem = mlp_train_smem();
    cudaError_t err = cudaFuncSetAttribute(mlp_train_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    mlp_train_kernel<<<ctas, kTB, smem, s>>>(feat, target, idx, batch, params, partial, loss_partial);
    reduce_grad_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(partial, ctas, grad);
    if (lr != 0.f) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
        adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, b1, b2, 1e-8f, bc1, bc2);
    }
    return cudaGetLastError();
}

}  // namespace mog
