// mog_device.cuh — device-side building blocks shared by the MOG kernels.
//
//  * per-(particle, grid) cell index in two arithmetic modes
//      FAST : t = (M^T/h) c + (L/2 - off)/h with fused multiply-adds, cell =
//             floor(t) mod g taken with one round-down add (mathematically the
//             cell of mass.glsl:42-50; may differ within ~1 ulp of a cell face)
//      EXACT: the shader's own sequence, mass.glsl:42-50 / update.glsl:71-74,
//             with IEEE-rounded mul/add/div and no contraction
//  * fixed-point mass quantisation (u64 scale 2^bits, or the reference's
//    uint(m * 1000.0) of mass.glsl:54)
//  * an in-register radix-2 DIT FFT of length 2..64 with the reference's
//    sign convention (fft_batched.glsl:19-34: forward e^{-i2pi kn/N},
//    inverse e^{+i2pi kn/N}, both unnormalised)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mog {

constexpr unsigned kFull = 0xffffffffu;

// Cell-index parameters of one grid, FAST mode: three rows (a0, a1, a2, b)
// so that t_r = a0*c.x + a1*c.y + a2*c.z + b with c = pos - L/2.
struct FastXf {
    float4 row[3];
};

// Everything a kernel needs to turn a position into a cell, per launch.
struct IndexParams {
    float half_l;     // L * 0.5 (mass.glsl:42)
    float world;      // L
    float voxel;      // h = L / g (main.py:118)
    int   lg;         // log2 g
};

// GLSL mod(x, y) = x - y * floor(x / y), with IEEE ops (mass.glsl:46).
__device__ __forceinline__ float glsl_mod(float x, float y) {
    return __fsub_rn(x, __fmul_rn(y, floorf(__fdiv_rn(x, y))));
}

// floor(t) mod 2^lg for |t| < 2^22: adding 1.5*2^23 with round-down leaves
// floor(t) in the low mantissa bits (the offset 2^22 is a multiple of g).
// NaN/Inf inputs give some index in [0, g), never an out-of-range one.
__device__ __forceinline__ uint32_t floor_mod_pow2(float t, uint32_t mask) {
    return __float_as_uint(__fadd_rd(t, 12582912.0f)) & mask;
}

// FAST mode cell index (x fastest, then y, then z), one grid.
__device__ __forceinline__ uint32_t cell_fast(const float4& r0, const float4& r1,
                                              const float4& r2, float cx, float cy,
                                              float cz, int lg) {
    const uint32_t mask = (1u << lg) - 1u;
    float tx = __fmaf_rn(r0.z, cz, __fmaf_rn(r0.y, cy, __fmaf_rn(r0.x, cx, r0.w)));
    float ty = __fmaf_rn(r1.z, cz, __fmaf_rn(r1.y, cy, __fmaf_rn(r1.x, cx, r1.w)));
    float tz = __fmaf_rn(r2.z, cz, __fmaf_rn(r2.y, cy, __fmaf_rn(r2.x, cx, r2.w)));
    uint32_t ix = floor_mod_pow2(tx, mask);
    uint32_t iy = floor_mod_pow2(ty, mask);
    uint32_t iz = floor_mod_pow2(tz, mask);
    return ix | (iy << lg) | (iz << (2 * lg));
}

// Slot of cell c = x | y << lg | z << 2 lg in a kFrameWorldSlot force grid:
// x XORed with (2y ^ 4z) mod 8 (and mod g).  A staged grid puts 8 cells
// (128 bytes) across the 32 banks, so cell c and its y and z neighbours
// (g and g^2 cells away, multiples of 8 for g >= 8) would share a 16-byte
// bank quad; with the slot, the cells of any 2 x 2 x 2 block sit in 8
// different quads.  x-rows and their aligned 8-cell blocks stay in place,
// so slabs and 128-byte lines are copied as before.  Its own inverse.
__host__ __device__ __forceinline__ uint32_t force_slot(uint32_t c, int lg) {
    const uint32_t mask = (1u << lg) - 1u;
    const uint32_t s = ((c >> (lg - 1)) & 6u) ^ ((c >> (2 * lg - 2)) & 4u);
    return c ^ (s & mask);
}

// force_slot of the cell whose x, y, z are the low lg bits of bx, by, bz
// (higher bits ignored).
__device__ __forceinline__ uint32_t force_slot_xyz(uint32_t bx, uint32_t by, uint32_t bz, int lg) {
    const uint32_t mask = (1u << lg) - 1u;
    const uint32_t x = (bx ^ (((by << 1) ^ (bz << 2)) & 7u)) & mask;
    return x | ((by & mask) << lg) | ((bz & mask) << (2 * lg));
}

// force_slot(cell_fast(...)).
__device__ __forceinline__ uint32_t slot_fast(const float4& r0, const float4& r1,
                                              const float4& r2, float cx, float cy,
                                              float cz, int lg) {
    const float tx = __fmaf_rn(r0.z, cz, __fmaf_rn(r0.y, cy, __fmaf_rn(r0.x, cx, r0.w)));
    const float ty = __fmaf_rn(r1.z, cz, __fmaf_rn(r1.y, cy, __fmaf_rn(r1.x, cx, r1.w)));
    const float tz = __fmaf_rn(r2.z, cz, __fmaf_rn(r2.y, cy, __fmaf_rn(r2.x, cx, r2.w)));
    return force_slot_xyz(__float_as_uint(__fadd_rd(tx, 12582912.0f)),
                          __float_as_uint(__fadd_rd(ty, 12582912.0f)),
                          __float_as_uint(__fadd_rd(tz, 12582912.0f)), lg);
}

// EXACT mode cell index.  R is the packed rotation of one grid,
// R[4j + r] = M[j][r]; the shader's mat3 has columns R[4j..4j+2], so
// rotated_r = (R[r]*c.x + R[4+r]*c.y) + R[8+r]*c.z  (GLSL mat3 * vec3).
__device__ __forceinline__ int exact_axis(float rot, float off, const IndexParams& ip,
                                          int g) {
    float l = __fsub_rn(__fadd_rn(rot, ip.half_l), off);          // mass.glsl:44
    l = glsl_mod(__fadd_rn(glsl_mod(l, ip.world), ip.world), ip.world);  // :46
    return __float2int_rz(__fdiv_rn(l, ip.voxel)) % g;            // :48-50
}

__device__ __forceinline__ uint32_t cell_exact(const float* R, const float* off,
                                               float cx, float cy, float cz,
                                               const IndexParams& ip) {
    const int g = 1 << ip.lg;
    float rx = __fadd_rn(__fadd_rn(__fmul_rn(R[0], cx), __fmul_rn(R[4], cy)), __fmul_rn(R[8], cz));
    float ry = __fadd_rn(__fadd_rn(__fmul_rn(R[1], cx), __fmul_rn(R[5], cy)), __fmul_rn(R[9], cz));
    float rz = __fadd_rn(__fadd_rn(__fmul_rn(R[2], cx), __fmul_rn(R[6], cy)), __fmul_rn(R[10], cz));
    int x = exact_axis(rx, off[0], ip, g);
    int y = exact_axis(ry, off[1], ip, g);
    int z = exact_axis(rz, off[2], ip, g);
    return (uint32_t)x | ((uint32_t)y << ip.lg) | ((uint32_t)z << (2 * ip.lg));
}

// World-frame vector M F of a grid-frame force, update.glsl:77
// (transpose(rot) * F with rot's columns R[4j..]):  out_r = (R[4r]F.x +
// R[4r+1]F.y) + R[4r+2]F.z, IEEE ops, no contraction.
__device__ __forceinline__ float3 rotate_back(const float* R, float fx, float fy, float fz) {
    float3 o;
    o.x = __fadd_rn(__fadd_rn(__fmul_rn(R[0], fx), __fmul_rn(R[1], fy)), __fmul_rn(R[2], fz));
    o.y = __fadd_rn(__fadd_rn(__fmul_rn(R[4], fx), __fmul_rn(R[5], fy)), __fmul_rn(R[6], fz));
    o.z = __fadd_rn(__fadd_rn(__fmul_rn(R[8], fx), __fmul_rn(R[9], fy)), __fmul_rn(R[10], fz));
    return o;
}

// ---- mass quantisation ------------------------------------------------
// u64: q = trunc(m * 2^bits); m*2^bits is exact in fp32 (power-of-two
// scale), so the truncation is exact.  Negative / NaN masses give 0 and
// raise BADMASS; values at or above 2^64 saturate and raise OVERFLOW.
__device__ __forceinline__ unsigned long long quantize_u64(float m, float scale,
                                                           unsigned& bad) {
    float v = __fmul_rn(m, scale);
    if (!(v >= 0.0f)) { bad |= 8u; return 0ull; }
    if (v >= 18446744073709551616.0f) { bad |= 2u; return ~0ull; }
    return __float2ull_rz(v);
}
// u32 x1000: uint(mass * 1000.0) (mass.glsl:54), saturating.
__device__ __forceinline__ unsigned quantize_u32(float m, unsigned& bad) {
    float v = __fmul_rn(m, 1000.0f);
    if (!(v >= 0.0f)) { bad |= 8u; return 0u; }
    if (v >= 4294967296.0f) return 0xffffffffu;
    return __float2uint_rz(v);
}
// Cell value as float: u64 -> round-to-nearest float * 2^-bits (exact
// scale); u32 -> float(v) / 1000.0 (complex.glsl:23).
__device__ __forceinline__ float mass_value(unsigned long long v, float inv_scale) {
    return __fmul_rn(__ull2float_rn(v), inv_scale);
}
__device__ __forceinline__ float mass_value(unsigned v, float) {
    return __fdiv_rn(__uint2float_rn(v), 1000.0f);
}

// ---- complex helpers ----------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// cos(2 pi j / 64) for j in [0, 64); first-quadrant values rounded from the
// exact ones, the rest by symmetry (so quarter points are exactly 0 / +-1).
__host__ __device__ constexpr float cos64(int j) {
    constexpr float q[17] = {
        1.000000000e+00f, 9.951847196e-01f, 9.807852507e-01f, 9.569403529e-01f,
        9.238795042e-01f, 8.819212914e-01f, 8.314695954e-01f, 7.730104327e-01f,
        7.071067691e-01f, 6.343932748e-01f, 5.555702448e-01f, 4.713967443e-01f,
        3.826834261e-01f, 2.902846634e-01f, 1.950903237e-01f, 9.801714122e-02f,
        0.0f};
    j &= 63;
    return j <= 16 ? q[j] : j <= 32 ? -q[32 - j] : j <= 48 ? -q[j - 32] : q[64 - j];
}
__host__ __device__ constexpr float sin64(int j) { return cos64(16 - j); }

template <int N>
__host__ __device__ constexpr int ilog2() {
    return N <= 1 ? 0 : 1 + ilog2<N / 2>();
}

template <int N>
__host__ __device__ constexpr int bitrev(int x) {
    int r = 0;
    for (int b = 0; b < ilog2<N>(); ++b) r = (r << 1) | ((x >> b) & 1);
    return r;
}

// In-register radix-2 DIT FFT, N in {1,2,4,...,64}.  Forward: X_k =
// sum_n x_n e^{-i 2 pi kn/N}; inverse: e^{+i...}, unnormalised.  The
// permutation, the butterflies and their twiddles are unrolled by template
// recursion, so every index and every twiddle is a compile-time constant
// and v stays in registers.  Twiddles of exactly 1 and -+i cost no
// multiplications.
namespace fftdetail {

template <int N, int I>
__device__ __forceinline__ void permute(float2 (&v)[N]) {
    if constexpr (I < N) {
        constexpr int r = bitrev<N>(I);
        if constexpr (r > I) {
            const float2 t = v[I];
            v[I] = v[r];
            v[r] = t;
        }
        permute<N, I + 1>(v);
    }
}

template <int N, bool INV, int S, int B, int J>
__device__ __forceinline__ void butterflies(float2 (&v)[N]) {
    if constexpr (B < N) {
        if constexpr (J < S / 2) {
            constexpr int H = S / 2;
            const float2 u = v[B + J];
            const float2 q = v[B + J + H];
            float2 wq;
            if constexpr (J == 0) {
                wq = q;
            } else if constexpr (4 * J == S) {
                wq = INV ? make_float2(-q.y, q.x) : make_float2(q.y, -q.x);
            } else {
                constexpr float c = cos64(J * (64 / S));
                constexpr float sn = INV ? sin64(J * (64 / S)) : -sin64(J * (64 / S));
                wq = make_float2(__fmaf_rn(q.x, c, -q.y * sn), __fmaf_rn(q.x, sn, q.y * c));
            }
            v[B + J] = cadd(u, wq);
            v[B + J + H] = csub(u, wq);
            butterflies<N, INV, S, B, J + 1>(v);
        } else {
            butterflies<N, INV, S, B + S, 0>(v);
        }
    }
}

template <int N, bool INV, int S>
__device__ __forceinline__ void stages(float2 (&v)[N]) {
    if constexpr (S <= N) {
        butterflies<N, INV, S, 0, 0>(v);
        stages<N, INV, 2 * S>(v);
    }
}

}  // namespace fftdetail

template <int N, bool INV>
__device__ __forceinline__ void fft_reg(float2 (&v)[N]) {
    static_assert(N >= 1 && N <= 64 && (N & (N - 1)) == 0, "fft length must be a power of two <= 64");
    fftdetail::permute<N, 0>(v);
    fftdetail::stages<N, INV, 2>(v);
}

// Status word helpers: raise bits once per warp.
__device__ __forceinline__ void raise_flags(unsigned* flags, unsigned bits) {
    unsigned any = __reduce_or_sync(__activemask(), bits);
    if (any && (threadIdx.x & 31) == __ffs(__activemask()) - 1) atomicOr(flags, any);
}

// Debug bounds check of a computed index i into a buffer of n elements.
// Built with -DMOG_CHECK, an index outside [0, n) raises MOG_FLAG_BOUNDS (16)
// in the status word and the caller skips the access, so a wrong index
// shows in mog_get_status instead of writing someone else's memory.
// Without it the check is the constant true and costs nothing.
#ifdef MOG_CHECK
__device__ __forceinline__ bool in_bounds(unsigned* flags, uint64_t i, uint64_t n) {
    if (i < n) return true;
    atomicOr(flags, 16u);
    return false;
}
#else
__device__ __forceinline__ constexpr bool in_bounds(unsigned*, uint64_t, uint64_t) { return true; }
#endif

}  // namespace mog
