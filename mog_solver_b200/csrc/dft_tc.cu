// dft_tc.cu — the 1-D DFT passes of the spectral solve on the tensor cores.
//
// With dft_prec = MOG_DFT_TC_BF16X3 every axis pass of the spectral solve
// (fft_batched.glsl:45-132, one per axis per transform) is a dense DFT
// written as a GEMM on the 5th-generation tensor cores (tcgen05):
//
//   D (128 lines x 2g reals) = A (128 lines x 2g reals) . B^T (2g x 2g)
//
// A row is one line of g complex values, (re, im) interleaved as they lie in
// memory; B is the real 2g x 2g form of the g-point DFT matrix W^(jl),
// W = exp(-+ 2 pi i / g):  row 2j (re out) = (cos, -sin) pairs, row 2j+1
// (im out) = (sin, cos) pairs.  FP32 inputs are split into BF16 hi + lo
// parts and three products are accumulated in FP32 in tensor memory:
//   D = A_hi B_hi + A_lo B_hi + A_hi B_lo
// (the lo x lo term, ~2^-16 relative, is dropped).  Forward and inverse are
// unnormalised, as in the FFT path; 1/g^3 is applied in the store.
//
// One CTA of 128 threads walks tiles of 128 lines: thread t converts line t
// into shared memory in the canonical K-major layout (core matrices of
// 8 rows x 16 bytes, no swizzle), one elected thread issues the MMAs and
// commits them to an mbarrier, and after the (bounded) wait every thread
// reads its own line's result from its TMEM lane and writes it back in
// place.  B (hi and lo, this pass's direction) stays in shared memory.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>

#include <cuda_bf16.h>

#include "mog_internal.h"

namespace mog {
namespace {

constexpr int kTileLines = 128;
constexpr long long kWaitCycles = 2000000000LL;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: no swizzle, K-major, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, dense.
constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                     uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask));
}

__device__ __forceinline__ void mbar_init(uint32_t addr) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(addr) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait on an mbarrier phase.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(addr, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

// 32 consecutive TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
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
}

__device__ __forceinline__ uint32_t bf16_pair(float lo_elem, float hi_elem) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// One axis pass over the lines of nf fields (f0, f1, f2; pairs x g^3
// complex each), in place.  axis 0: x (contiguous), 1: y (stride g),
// 2: z (stride g^2).  tables: B hi, B lo for the forward direction, then
// for the inverse, each (2g)^2 BF16 in the canonical layout.
template <int G>
__global__ void __launch_bounds__(kTileLines) dft_tc_kernel(float2* f0, float2* f1, float2* f2,
                                                            int nf, int axis, int pairs, int inv,
                                                            const uint4* __restrict__ tables,
                                                            unsigned* flags) {
    constexpr int KD = 2 * G;                  // reals per line: K = N of the GEMM
    constexpr int KB = KD / 8;                 // 16-byte k-blocks per row
    constexpr uint32_t LBO = 128;              // next k-block
    constexpr uint32_t SBO = KB * 128;         // next 8-row group
    constexpr uint32_t ABYTES = kTileLines * KD * 2;
    constexpr uint32_t BBYTES = KD * KD * 2;
    constexpr uint32_t NCOLS = KD < 32 ? 32 : KD;
    constexpr int G3 = G * G * G;
    static_assert(KD % 32 == 0, "whole 32-column TMEM loads");
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* a_hi = sm;
    unsigned char* a_lo = sm + ABYTES;
    unsigned char* b_hi = sm + 2 * ABYTES;
    unsigned char* b_lo = b_hi + BBYTES;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;

    {
        const uint4* src = tables + (size_t)(inv ? 2 : 0) * (BBYTES / 16);
        uint4* dst = reinterpret_cast<uint4*>(b_hi);
        for (int i = t; i < (int)(2 * BBYTES / 16); i += kTileLines) dst[i] = src[i];
    }
    const uint32_t mbar_addr = smem_u32(&mbar);
    if (t == 0) mbar_init(mbar_addr);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(NCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t a_hi_s = smem_u32(a_hi), a_lo_s = smem_u32(a_lo);
    const uint32_t b_hi_s = smem_u32(b_hi), b_lo_s = smem_u32(b_lo);
    const uint32_t row_off = (uint32_t)(t >> 3) * SBO + (uint32_t)(t & 7) * 16;

    const int64_t per_field = (int64_t)pairs * G * G;
    const int64_t lines = per_field * nf;
    const int64_t tiles = (lines + kTileLines - 1) / kTileLines;
    uint32_t parity = 0;
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t line = tile * kTileLines + t;
        const bool live = line < lines;
        float2* p = f0;
        int64_t stride = 1;
        if (live) {
            const int f = (int)(line / per_field);
            const int64_t rem = line % per_field;
            const int64_t pair = rem / (G * G);
            const int r = (int)(rem % (G * G));
            float2* buf = f == 0 ? f0 : (f == 1 ? f1 : f2);
            int64_t base;
            if (axis == 0) {
                base = (int64_t)r * G;
                stride = 1;
            } else if (axis == 1) {
                base = (int64_t)(r / G) * G * G + (r % G);
                stride = G;
            } else {
                base = r;
                stride = (int64_t)G * G;
            }
            p = buf + pair * G3 + base;
        }
        // line t -> registers (all loads in flight; 16-byte loads along x)
        float2 v[G];
        if (live && stride == 1) {
            const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
            for (int j = 0; j < G / 2; ++j) {
                const float4 a = q[j];
                v[2 * j] = make_float2(a.x, a.y);
                v[2 * j + 1] = make_float2(a.z, a.w);
            }
        } else {
#pragma unroll
            for (int j = 0; j < G; ++j) v[j] = live ? p[(int64_t)j * stride] : make_float2(0.f, 0.f);
        }
        // -> row t of A (hi and lo), 4 complex values per k-block
#pragma unroll
        for (int kb = 0; kb < KB; ++kb) {
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 x = v[kb * 4 + j];
                const __nv_bfloat16 hr = __float2bfloat16_rn(x.x), hi_ = __float2bfloat16_rn(x.y);
                hi[j] = bf16_pair(__bfloat162float(hr), __bfloat162float(hi_));
                lo[j] = bf16_pair(x.x - __bfloat162float(hr), x.y - __bfloat162float(hi_));
            }
            const uint32_t off = row_off + (uint32_t)kb * LBO;
            *reinterpret_cast<uint4*>(a_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4*>(a_lo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t idesc = instr_desc(kTileLines, KD);
            uint32_t acc = 0;
#pragma unroll
            for (int part = 0; part < 3; ++part) {
                const uint32_t a = part == 1 ? a_lo_s : a_hi_s;
                const uint32_t b = part == 2 ? b_lo_s : b_hi_s;
#pragma unroll
                for (int s = 0; s < KD / 16; ++s) {
                    umma(tmem, smem_desc(a + 256u * s, LBO, SBO), smem_desc(b + 256u * s, LBO, SBO),
                         idesc, acc);
                    acc = 1;
                }
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    mbar_addr)
                : "memory");
        }
        const bool done = mbar_wait(mbar_addr, parity);
        ok = __syncthreads_and(done) != 0;
        if (!ok) break;
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int c = 0; c < KD; c += 32) {
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
            if (live && stride == 1) {
                float4* q = reinterpret_cast<float4*>(p) + c / 4;
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    q[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                       __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
            } else if (live) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    p[(int64_t)(c / 2 + j) * stride] =
                        make_float2(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]));
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // TMEM and the A tiles are free for the next tile
    }
    if (!ok) {
        // the MMAs of the last tile did not complete in time: report, give
        // them one more bounded wait, then release the tensor memory
        if (t == 0) atomicOr(flags, 4u);  // MOG_FLAG_TIMEOUT
        mbar_wait(mbar_addr, parity);
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS)
                     : "memory");
    }
}

uint16_t bf16_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t rounding = 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
    return (uint16_t)((u + rounding) >> 16);
}

float bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

}  // namespace

// Host: B hi / lo of the forward and inverse g-point DFT in the canonical
// layout the kernel's descriptors describe: element (n, k) of the 2g x 2g
// real matrix at byte (n / 8) * (2g / 8) * 128 + (k / 8) * 128 + (n % 8) * 16
// + (k % 8) * 2.  Angles in FP64.
std::vector<uint16_t> dft_tc_tables(int g) {
    const int KD = 2 * g, KB = KD / 8;
    const size_t per = (size_t)KD * KD;
    std::vector<uint16_t> out(4 * per);
    const double two_pi = 6.283185307179586476925286766559;
    for (int dir = 0; dir < 2; ++dir) {
        const double sgn = dir == 0 ? -1.0 : 1.0;
        for (int n = 0; n < KD; ++n)
            for (int k = 0; k < KD; ++k) {
                const int j = n / 2, l = k / 2;
                const double th = sgn * two_pi * (double)((j * l) % g) / (double)g;
                const double c = std::cos(th), s = std::sin(th);
                double v;
                if ((n & 1) == 0) v = (k & 1) == 0 ? c : -s;
                else v = (k & 1) == 0 ? s : c;
                const float f = (float)v;
                const uint16_t hb = bf16_bits(f);
                const uint16_t lb = bf16_bits((float)(v - (double)bf16_value(hb)));
                const size_t idx = (size_t)(n / 8) * KB * 64 + (size_t)(k / 8) * 64 + (n % 8) * 8 + (k % 8);
                out[(size_t)(2 * dir) * per + idx] = hb;
                out[(size_t)(2 * dir + 1) * per + idx] = lb;
            }
    }
    return out;
}

size_t dft_tc_smem(int g) {
    const size_t KD = 2 * (size_t)g;
    return 2 * (size_t)kTileLines * KD * 2 + 2 * KD * KD * 2;
}

cudaError_t launch_dft_tc(int g, float2* f0, float2* f1, float2* f2, int nf, int axis, int pairs,
                          bool inverse, const void* tables, unsigned* flags, cudaStream_t s) {
    const int64_t lines = (int64_t)nf * pairs * g * g;
    const int64_t tiles = (lines + kTileLines - 1) / kTileLines;
    const size_t smem = dft_tc_smem(g);
    auto go = [&](auto kern) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (err != cudaSuccess) return err;
        int per_sm = 0;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileLines, smem);
        if (err != cudaSuccess) return err;
        const int64_t blocks = std::min<int64_t>(tiles, (int64_t)num_sms() * std::max(per_sm, 1));
        kern<<<(unsigned)blocks, kTileLines, smem, s>>>(f0, f1, f2, nf, axis, pairs, inverse ? 1 : 0,
                                                       static_cast<const uint4*>(tables), flags);
        return cudaGetLastError();
    };
    if (g == 16) return go(dft_tc_kernel<16>);
    if (g == 32) return go(dft_tc_kernel<32>);
    return cudaErrorInvalidValue;
}

}  // namespace mog
