// learned.cu — learned correction of a cheap MOG ensemble.
//
// No counterpart in the reference: its force is always the plain average
// over k grids (update.glsl:67-81).  Here a small network (12 -> 64 -> 64 -> 3,
// GELU) predicts, from statistics of a cheap ensemble (k = 32), the residual
// to an expensive one (k = 240):
//
//   features  per particle, from the k grids it touches: the mean world
//             force, a least-squares correction of it from the particle's
//             offsets to its cells' centres, the per-grid force spread, the
//             mean cell mass and two scalars (see features_kernel);
//             standardised with the model's statistics;
//   inference BF16 tensor-core MLP (mma.sync m16n8k16, FP32 accumulate).
//             A warp carries 16 particles through all three layers in
//             registers: the accumulator fragment of one layer is, pair of
//             n-tiles by pair, exactly the A fragment of the next;
//   training  FP32 fused forward + backward over a minibatch, one CTA per
//             128 samples, per-CTA partial gradients reduced in a fixed
//             order (deterministic), then Adam.
//
// Parameter vector layout (FP32, kParams floats):
//   W1[64][12] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>

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
// Inference: the hardware tanh approximation (relative error ~2^-11, far
// below BF16 resolution).
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_fast(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanh_fast(u));
}

// ---------------------------------------------------------------------------
// Feature gather.  One thread per particle; grids read from L2.
//
// Each grid samples the force at the centre of the particle's cell, not at
// the particle, so the k per-grid forces F_i scatter around the force at
// the particle roughly linearly in the particle's offset from those cell
// centres, d_i (world frame).  A per-particle least-squares fit
// F_i ~ a + B d_i over the k grids gives an intercept a, the force
// extrapolated to the particle itself:
//     a = Fbar - C_Fd (C_dd + ridge)^-1 dbar
// with dbar, C_dd = cov(d, d) and C_Fd = cov(F, d) over the grids.
// The features are
//   0-2  Fbar / s            plain ensemble mean (update.glsl order)
//   3-5  (a - Fbar) / s      regression correction from the in-cell offsets
//   6-8  std_i(F_i) / s      per-component spread of the per-grid forces
//   9    log1p(rho / rho_ref) mean mass of the particle's cells
//   10   |Fbar| / s
//   11   sqrt(tr C_dd) / h   spread of the in-cell offsets
// then standardised with the model's mu / sigma; slots 12-14 carry the
// regression correction a - Fbar itself (world units, not standardised;
// the first layer's weights for slots 12-15 are zero) and slot 15 is 0.
template <typename Acc>
__global__ void __launch_bounds__(256) features_kernel(const float4* __restrict__ pos, int64_t n,
                                                       const float4* __restrict__ W,
                                                       const Acc* __restrict__ mass, Ensemble e,
                                                       ModelNorm norm, float4* __restrict__ mean_out,
                                                       float* __restrict__ feat_out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const IndexParams ip = e.index_params();
    const float4 P = pos[p];
    const float cx = __fsub_rn(P.x, ip.half_l), cy = __fsub_rn(P.y, ip.half_l),
                cz = __fsub_rn(P.z, ip.half_l);
    const int G3 = 1 << (3 * e.lg);
    const uint32_t mask = (1u << e.lg) - 1u;
    const float h = e.voxel;
    float sx = 0.f, sy = 0.f, sz = 0.f;            // plain sum, update.glsl order
    float qx = 0.f, qy = 0.f, qz = 0.f;            // sum F^2 per component
    float dx = 0.f, dy = 0.f, dz = 0.f;            // sum d
    float dxx = 0.f, dxy = 0.f, dxz = 0.f, dyy = 0.f, dyz = 0.f, dzz = 0.f;
    float fxdx = 0.f, fxdy = 0.f, fxdz = 0.f, fydx = 0.f, fydy = 0.f, fydz = 0.f,
          fzdx = 0.f, fzdy = 0.f, fzdz = 0.f;      // sum F d^T
    float rho = 0.f;
    for (int i = 0; i < e.k; ++i) {
        const FastXf x = e.fast[i];
        const float tx = __fmaf_rn(x.row[0].z, cz, __fmaf_rn(x.row[0].y, cy, __fmaf_rn(x.row[0].x, cx, x.row[0].w)));
        const float ty = __fmaf_rn(x.row[1].z, cz, __fmaf_rn(x.row[1].y, cy, __fmaf_rn(x.row[1].x, cx, x.row[1].w)));
        const float tz = __fmaf_rn(x.row[2].z, cz, __fmaf_rn(x.row[2].y, cy, __fmaf_rn(x.row[2].x, cx, x.row[2].w)));
        uint32_t c;
        if (e.index_mode == 0)
            c = floor_mod_pow2(tx, mask) | (floor_mod_pow2(ty, mask) << e.lg) |
                (floor_mod_pow2(tz, mask) << (2 * e.lg));
        else
            c = cell_exact(e.rot12 + 12 * i, e.off4 + 4 * i, cx, cy, cz, ip);
        const float4 f = __ldg(W + (size_t)i * G3 + c);
        sx = __fadd_rn(sx, f.x);
        sy = __fadd_rn(sy, f.y);
        sz = __fadd_rn(sz, f.z);
        qx += f.x * f.x;
        qy += f.y * f.y;
        qz += f.z * f.z;
        // offset from the cell centre, grid frame -> world frame (M d)
        const float gx = (tx - floorf(tx) - 0.5f) * h, gy = (ty - floorf(ty) - 0.5f) * h,
                    gz = (tz - floorf(tz) - 0.5f) * h;
        const float* R = e.rot12 + 12 * i;
        const float wx = R[0] * gx + R[1] * gy + R[2] * gz;
        const float wy = R[4] * gx + R[5] * gy + R[6] * gz;
        const float wz = R[8] * gx + R[9] * gy + R[10] * gz;
        dx += wx; dy += wy; dz += wz;
        dxx += wx * wx; dxy += wx * wy; dxz += wx * wz;
        dyy += wy * wy; dyz += wy * wz; dzz += wz * wz;
        fxdx += f.x * wx; fxdy += f.x * wy; fxdz += f.x * wz;
        fydx += f.y * wx; fydy += f.y * wy; fydz += f.y * wz;
        fzdx += f.z * wx; fzdy += f.z * wy; fzdz += f.z * wz;
        rho += mass_value(__ldg(mass + (size_t)i * G3 + c), e.inv_scale);
    }
    const float kf = (float)e.k, ik = 1.0f / kf;
    const float mx = __fdiv_rn(sx, kf), my = __fdiv_rn(sy, kf), mz = __fdiv_rn(sz, kf);
    mean_out[p] = make_float4(mx, my, mz, 0.f);
    const float ax_ = dx * ik, ay_ = dy * ik, az_ = dz * ik;  // dbar
    // covariances
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
        const float id = 1.0f / det;
        wx = (A00 * ax_ + A01 * ay_ + A02 * az_) * id;
        wy = (A01 * ax_ + A11 * ay_ + A12 * az_) * id;
        wz = (A02 * ax_ + A12 * ay_ + A22 * az_) * id;
    }
    // correction = -C_Fd w,  C_Fd = sum(F d^T)/k - Fbar dbar^T
    const float ex = -((fxdx * ik - mx * ax_) * wx + (fxdy * ik - mx * ay_) * wy + (fxdz * ik - mx * az_) * wz);
    const float ey = -((fydx * ik - my * ax_) * wx + (fydy * ik - my * ay_) * wy + (fydz * ik - my * az_) * wz);
    const float ez = -((fzdx * ik - mz * ax_) * wx + (fzdy * ik - mz * ay_) * wy + (fzdz * ik - mz * az_) * wz);
    const float is = 1.0f / norm.force_scale;
    float f[kIn];
    f[0] = mx * is;
    f[1] = my * is;
    f[2] = mz * is;
    f[3] = ex * is;
    f[4] = ey * is;
    f[5] = ez * is;
    f[6] = sqrtf(fmaxf(qx * ik - mx * mx, 0.f)) * is;
    f[7] = sqrtf(fmaxf(qy * ik - my * my, 0.f)) * is;
    f[8] = sqrtf(fmaxf(qz * ik - mz * mz, 0.f)) * is;
    f[9] = log1pf(rho * ik / norm.rho_ref);
    f[10] = sqrtf(mx * mx + my * my + mz * mz) * is;
    f[11] = sqrtf(fmaxf(cxx + cyy + czz - 3.f * ridge, 0.f)) / h;
    float* o = feat_out + (size_t)p * 16;
#pragma unroll
    for (int j = 0; j < kIn; ++j) o[j] = (f[j] - norm.mu[j]) * norm.inv_sigma[j];
    o[12] = ex;
    o[13] = ey;
    o[14] = ez;
    o[15] = 0.f;
}

// ---------------------------------------------------------------------------
// BF16 weight fragments for mma.sync.m16n8k16 (B operand, "col" layout):
// for k-step ks and n-tile nt, lane l holds
//   b0 = {W[n][k], W[n][k+1]} with n = nt*8 + l/4, k = ks*16 + 2*(l%4)
//   b1 = the same at k + 8.
// Stored as uint2 [ks][nt][32] so a warp reads 256 contiguous bytes.
constexpr int kFrag1 = 1 * 8, kFrag2 = 4 * 8, kFrag3 = 4 * 1;  // (k-steps x n-tiles)
constexpr int kFragTotal = (kFrag1 + kFrag2 + kFrag3) * 32;     // uint2 per model

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
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
    auto w = [&](int nn, int kk) { return (nn < out && kk < in) ? Wm[nn * in + kk] : 0.f; };
    frags[t] = make_uint2(pack_bf16(w(n, k), w(n, k + 1)), pack_bf16(w(n, k + 8), w(n, k + 9)));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Tensor-core inference.  Each warp owns 16 consecutive particles (one
// m16 tile).  Output: acc[p] = base + out_scale * y  (the corrected
// ensemble force), written for the update to apply; base is mean[p], or
// mean[p] + the regression correction (feature slots 12-14) when
// with_correction is set.
__global__ void __launch_bounds__(128) mlp_infer_kernel(const float* __restrict__ feat, int64_t n,
                                                        const uint2* __restrict__ frags,
                                                        const float* __restrict__ params,
                                                        const float4* __restrict__ mean,
                                                        float out_scale, bool with_correction,
                                                        float4* __restrict__ acc) {
    __shared__ uint2 sf[kFragTotal];
    __shared__ float sb[kH + kH + 8];
    for (int i = threadIdx.x; i < kFragTotal; i += blockDim.x) sf[i] = frags[i];
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        sb[i] = params[kB1 + i];
        sb[kH + i] = params[kB2 + i];
    }
    if (threadIdx.x < 8) sb[2 * kH + threadIdx.x] = threadIdx.x < kOut ? params[kB3 + threadIdx.x] : 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
         tile * 16 < n; tile += warps) {
        const int64_t r0 = tile * 16 + g, r1 = r0 + 8;
        // layer 1 A fragment straight from the feature rows (16 floats each)
        auto ld2 = [&](int64_t r, int c) -> uint32_t {
            if (r >= n) return 0u;
            const float2 v = *reinterpret_cast<const float2*>(feat + r * 16 + c);
            return pack_bf16(v.x, v.y);
        };
        const uint32_t a0 = ld2(r0, 2 * tg), a1 = ld2(r1, 2 * tg), a2 = ld2(r0, 2 * tg + 8),
                       a3 = ld2(r1, 2 * tg + 8);
        float h[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float b0 = sb[nt * 8 + 2 * tg], b1 = sb[nt * 8 + 2 * tg + 1];
            h[nt][0] = b0; h[nt][1] = b1; h[nt][2] = b0; h[nt][3] = b1;
            const uint2 w = sf[(0 * 8 + nt) * 32 + lane];
            mma_bf16(h[nt], a0, a1, a2, a3, w.x, w.y);
        }
        uint32_t A[4][4];
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            A[ks][0] = pack_bf16(gelu_fast(h[2 * ks][0]), gelu_fast(h[2 * ks][1]));
            A[ks][1] = pack_bf16(gelu_fast(h[2 * ks][2]), gelu_fast(h[2 * ks][3]));
            A[ks][2] = pack_bf16(gelu_fast(h[2 * ks + 1][0]), gelu_fast(h[2 * ks + 1][1]));
            A[ks][3] = pack_bf16(gelu_fast(h[2 * ks + 1][2]), gelu_fast(h[2 * ks + 1][3]));
        }
        // layer 2
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float b0 = sb[kH + nt * 8 + 2 * tg], b1 = sb[kH + nt * 8 + 2 * tg + 1];
            h[nt][0] = b0; h[nt][1] = b1; h[nt][2] = b0; h[nt][3] = b1;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint2 w = sf[(kFrag1 + ks * 8 + nt) * 32 + lane];
                mma_bf16(h[nt], A[ks][0], A[ks][1], A[ks][2], A[ks][3], w.x, w.y);
            }
        }
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            A[ks][0] = pack_bf16(gelu_fast(h[2 * ks][0]), gelu_fast(h[2 * ks][1]));
            A[ks][1] = pack_bf16(gelu_fast(h[2 * ks][2]), gelu_fast(h[2 * ks][3]));
            A[ks][2] = pack_bf16(gelu_fast(h[2 * ks + 1][0]), gelu_fast(h[2 * ks + 1][1]));
            A[ks][3] = pack_bf16(gelu_fast(h[2 * ks + 1][2]), gelu_fast(h[2 * ks + 1][3]));
        }
        // layer 3 (n = 8, outputs 0..2 live)
        float y[4];
        y[0] = sb[2 * kH + 2 * tg];
        y[1] = sb[2 * kH + 2 * tg + 1];
        y[2] = y[0];
        y[3] = y[1];
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const uint2 w = sf[(kFrag1 + kFrag2 + ks) * 32 + lane];
            mma_bf16(y, A[ks][0], A[ks][1], A[ks][2], A[ks][3], w.x, w.y);
        }
        // lanes with tg == 0 hold outputs 0,1 of rows g, g+8; tg == 1 holds output 2
        const float o0a = __shfl_sync(kFull, y[0], (g << 2) | 0), o1a = __shfl_sync(kFull, y[1], (g << 2) | 0);
        const float o2a = __shfl_sync(kFull, y[0], (g << 2) | 1);
        const float o0b = __shfl_sync(kFull, y[2], (g << 2) | 0), o1b = __shfl_sync(kFull, y[3], (g << 2) | 0);
        const float o2b = __shfl_sync(kFull, y[2], (g << 2) | 1);
        auto base = [&](int64_t r) {
            float4 m = mean[r];
            if (with_correction) {
                const float4 c = *reinterpret_cast<const float4*>(feat + r * 16 + 12);
                m.x += c.x;
                m.y += c.y;
                m.z += c.z;
            }
            return m;
        };
        if (tg == 0) {
            if (r0 < n) {
                const float4 m = base(r0);
                acc[r0] = make_float4(m.x + out_scale * o0a, m.y + out_scale * o1a, m.z + out_scale * o2a, 0.f);
            }
            if (r1 < n) {
                const float4 m = base(r1);
                acc[r1] = make_float4(m.x + out_scale * o0b, m.y + out_scale * o1b, m.z + out_scale * o2b, 0.f);
            }
        }
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

// Apply a per-particle force with the update.glsl:83-89 arithmetic.
__global__ void apply_force_kernel(float4* __restrict__ pos, float4* __restrict__ vel, int64_t n,
                                   const float4* __restrict__ acc, float dt, float damp,
                                   float world, unsigned* flags) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 P = pos[p], V = vel[p], A = acc[p];
    float vx = __fmul_rn(__fsub_rn(V.x, __fmul_rn(A.x, dt)), damp);
    float vy = __fmul_rn(__fsub_rn(V.y, __fmul_rn(A.y, dt)), damp);
    float vz = __fmul_rn(__fsub_rn(V.z, __fmul_rn(A.z, dt)), damp);
    const float px = glsl_mod(__fadd_rn(P.x, __fmul_rn(vx, dt)), world);
    const float py = glsl_mod(__fadd_rn(P.y, __fmul_rn(vy, dt)), world);
    const float pz = glsl_mod(__fadd_rn(P.z, __fmul_rn(vz, dt)), world);
    if (!(isfinite(px) && isfinite(py) && isfinite(pz))) atomicOr(flags, 1u);
    pos[p] = make_float4(px, py, pz, P.w);
    vel[p] = make_float4(vx, vy, vz, 0.f);
}

}  // namespace

int mlp_param_count() { return kParams; }
size_t mlp_fragment_bytes() { return sizeof(uint2) * kFragTotal; }
size_t mlp_train_smem() {
    return sizeof(float) * ((size_t)kParams + kTB * kIn + 4 * kTB * kLd + kTB * 4);
}

cudaError_t launch_features(const Ensemble& e, const float4* pos, int64_t n, const float4* W,
                            const void* mass, const ModelNorm& norm, float4* mean, float* feat,
                            cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (e.mass_mode == 0)
        features_kernel<unsigned long long><<<blocks, 256, 0, s>>>(
            pos, n, W, static_cast<const unsigned long long*>(mass), e, norm, mean, feat);
    else
        features_kernel<unsigned><<<blocks, 256, 0, s>>>(pos, n, W, static_cast<const unsigned*>(mass),
                                                         e, norm, mean, feat);
    return cudaGetLastError();
}

cudaError_t launch_pack_fragments(const float* params, void* frags, cudaStream_t s) {
    pack_fragments_kernel<<<(kFragTotal + 255) / 256, 256, 0, s>>>(params, static_cast<uint2*>(frags));
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const float* feat, int64_t n, const void* frags, const float* params,
                             const float4* mean, float out_scale, bool with_correction, float4* acc,
                             cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int64_t tiles = (n + 15) / 16;
    const int64_t blocks = std::min<int64_t>((tiles + 3) / 4, (int64_t)num_sms() * 16);
    mlp_infer_kernel<<<(unsigned)blocks, 128, 0, s>>>(feat, n, static_cast<const uint2*>(frags),
                                                      params, mean, out_scale, with_correction, acc);
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

cudaError_t launch_apply_force(float4* pos, float4* vel, int64_t n, const float4* acc, float dt,
                               float damp, float world, unsigned* flags, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    apply_force_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pos, vel, n, acc, dt, damp, world, flags);
    return cudaGetLastError();
}

}  // namespace mog
