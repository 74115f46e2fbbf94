// convolution.cu — `solver: convolution`: direct real-space force per grid.
//
// The reference parses `solver: fft|convolution` (main.py:125-126) and
// builds a real-space kernel K(d) = r/(4 pi |r|^3) on minimum-image cell
// offsets (main.py:250-278), but no shader ever binds it and step()
// always runs the FFT chain (main.py:671-672).  Here the switch is real:
//     F_i(x) = 2 pi G h^3 * sum_y m_i(y) K((x - y) mod g)
// with the reference's kernel table, scaled so that both solvers produce
// forces in the same units (the FFT chain's output is h^3/2 times the
// Newtonian periodic field for G: -2 pi instead of -4 pi in greens.glsl:40,
// cell mass instead of density, and 1/g^3 instead of 1/L^3 in pack.glsl:21).
// Minimum-image summation neither subtracts the mean density nor adds
// periodic images, so the two solvers agree at short range only.
//
// One CTA per grid: the grid's cell masses are read once into shared
// memory as floats and every thread sums over the non-empty source cells
// (the branch is warp-uniform: all lanes visit the same source).
#include "mog_internal.h"

namespace mog {

namespace {

template <typename Acc>
__global__ void __launch_bounds__(1024) conv_kernel(const Acc* __restrict__ mass,
                                                    float4* __restrict__ force, Ensemble e,
                                                    float coef, int frame) {
    extern __shared__ float msm[];
    const int lg = e.lg, g = 1 << lg;
    const int G3 = 1 << (3 * lg);
    const int i = blockIdx.x;
    const Acc* m = mass + (size_t)i * G3;
    for (int c = threadIdx.x; c < G3; c += blockDim.x) msm[c] = mass_value(m[c], e.inv_scale);
    __syncthreads();
    float R[12];
    for (int q = 0; q < 12; ++q) R[q] = __ldg(e.rot12 + 12 * i + q);
    const int mask = g - 1;
    for (int t = threadIdx.x; t < G3; t += blockDim.x) {
        const int tx = t & mask, ty = (t >> lg) & mask, tz = t >> (2 * lg);
        float fx = 0.f, fy = 0.f, fz = 0.f;
        for (int s = 0; s < G3; ++s) {
            const float ms = msm[s];
            if (ms == 0.f) continue;
            const int dx = (tx - (s & mask)) & mask;
            const int dy = (ty - ((s >> lg) & mask)) & mask;
            const int dz = (tz - (s >> (2 * lg))) & mask;
            const float4 K = __ldg(e.conv_kernel + (((dz << lg) | dy) << lg | dx));
            fx = __fmaf_rn(ms, K.x, fx);
            fy = __fmaf_rn(ms, K.y, fy);
            fz = __fmaf_rn(ms, K.z, fz);
        }
        fx *= coef;
        fy *= coef;
        fz *= coef;
        float4 out;
        if (frame != kFrameGrid) {
            const float3 w = rotate_back(R, fx, fy, fz);
            out = make_float4(w.x, w.y, w.z, 0.f);
        } else {
            out = make_float4(fx, fy, fz,
                              __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)),
                                                   __fmul_rn(fz, fz))));
        }
        force[(size_t)i * G3 + (frame == kFrameWorldSlot ? force_slot((uint32_t)t, lg) : (uint32_t)t)] = out;
    }
}

__global__ void conv_check_total_kernel(Ensemble e) {
    if (e.mass_mode == 0 && e.mass_total) {
        if (*e.mass_total >= 18446744073709551616.0) atomicOr(e.flags, 2u);
        *e.mass_total = 0.0;
    }
}

}  // namespace

cudaError_t launch_convolution(const Ensemble& e, void* mass, float4* force, int frame,
                               bool zero_mass, cudaStream_t s) {
    if (frame < kFrameGrid || frame > kFrameWorldSlot) return cudaErrorInvalidValue;
    const int G3 = 1 << (3 * e.lg);
    const size_t smem = (size_t)G3 * sizeof(float);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;  // g <= 32
    const double h = (double)e.voxel;
    const float coef = (float)(2.0 * 3.14159265358979323846 * (double)e.G * h * h * h);
    const int threads = 1024;
    if (zero_mass) conv_check_total_kernel<<<1, 1, 0, s>>>(e);
    cudaError_t err;
    if (e.mass_mode == 0) {
        auto kern = conv_kernel<unsigned long long>;
        err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        kern<<<e.k, threads, smem, s>>>(static_cast<unsigned long long*>(mass), force, e, coef,
                                        frame);
    } else {
        auto kern = conv_kernel<unsigned>;
        err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        kern<<<e.k, threads, smem, s>>>(static_cast<unsigned*>(mass), force, e, coef,
                                        frame);
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    if (zero_mass) {
        const size_t bytes = (size_t)e.cells() * (e.mass_mode == 0 ? 8 : 4);
        err = cudaMemsetAsync(mass, 0, bytes, s);
    }
    return err;
}

}  // namespace mog
