// diagnostics.cu — FP64 direct-sum yardstick of force accuracy.
//
// The accuracy half of the headline metric compares MOG forces with an FP64
// direct sum.  The reference has no such tool; its paper reports a 2-D MSE
// from a script that is not shipped.  In the solver's units the reference's
// field is (h^3 / 2) times the Newtonian periodic gradient for G: -2 pi G
// instead of -4 pi G in greens.glsl:40, cell masses instead of densities,
// and 1/g^3 instead of 1/L^3 in pack.glsl:21.  So the yardstick sums
//     F(x) = g_eff * sum_j m_j d / (|d|^2 + soft^2)^(3/2),
//     d = minimum-image (x - x_j),  g_eff = G h^3 / 2,
// which points away from the sources like the solver's F (update.glsl:83
// subtracts it).  Sources are tiled through shared memory in FP64; each
// target accumulates the sources of one chunk, and the chunks' partial sums
// are added in a fixed order, so the result is deterministic.
#include <mutex>

#include "mog_internal.h"

namespace mog {

namespace {

constexpr int kTile = 512;

__global__ void __launch_bounds__(128) direct_partial_kernel(
    const float4* __restrict__ targets, int64_t nt, const float4* __restrict__ sources, int64_t ns,
    int64_t per_chunk, double world, double g_eff, double soft2, double* __restrict__ partial) {
    __shared__ double4 tile[kTile];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    const int64_t s0 = (int64_t)chunk * per_chunk;
    const int64_t s1 = min(ns, s0 + per_chunk);
    double tx = 0, ty = 0, tz = 0;
    if (t < nt) {
        const float4 T = targets[t];
        tx = T.x;
        ty = T.y;
        tz = T.z;
    }
    const double inv_l = 1.0 / world;
    double fx = 0, fy = 0, fz = 0;
    for (int64_t base = s0; base < s1; base += kTile) {
        const int cnt = (int)(s1 - base < kTile ? s1 - base : kTile);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            const float4 S = sources[base + i];
            tile[i] = make_double4(S.x, S.y, S.z, S.w);
        }
        __syncthreads();
        if (t < nt) {
            for (int i = 0; i < cnt; ++i) {
                const double4 S = tile[i];
                double dx = tx - S.x, dy = ty - S.y, dz = tz - S.z;
                dx -= world * rint(dx * inv_l);
                dy -= world * rint(dy * inv_l);
                dz -= world * rint(dz * inv_l);
                const double r2 = dx * dx + dy * dy + dz * dz + soft2;
                if (r2 > 0.0) {
                    const double inv = 1.0 / (r2 * sqrt(r2));
                    const double w = S.w * inv;
                    fx += w * dx;
                    fy += w * dy;
                    fz += w * dz;
                }
            }
        }
    }
    if (t < nt) {
        double* o = partial + ((size_t)chunk * nt + t) * 3;
        o[0] = g_eff * fx;
        o[1] = g_eff * fy;
        o[2] = g_eff * fz;
    }
}

__global__ void direct_reduce_kernel(const double* __restrict__ partial, int64_t nt, int chunks,
                                     double* __restrict__ out3) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt * 3) return;
    double s = 0;
    for (int c = 0; c < chunks; ++c) s += partial[(size_t)c * nt * 3 + i];
    out3[i] = s;
}

// Fixed scratch of mog_direct_sum_noalloc: the per-chunk partial sums of up
// to kDirectScratchPairs (target, chunk) pairs, 3 doubles each (12 MiB).
// One copy exists on every device the library runs on.
__device__ __align__(256) static double g_direct_scratch[3 * kDirectScratchPairs];

}  // namespace

// Device address of g_direct_scratch on the current device, looked up once
// per device (cudaGetSymbolAddress, with that device current) and cached.
cudaError_t direct_sum_scratch(double** out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static double* addr[kMaxDevices] = {};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_direct_scratch);
        if (err != cudaSuccess) return err;
        addr[dev] = static_cast<double*>(p);
    }
    *out = addr[dev];
    return cudaSuccess;
}

cudaError_t launch_direct_sum(const float4* targets, int64_t nt, const float4* sources, int64_t ns,
                              double world, double g_eff, double soft, double* partial, int chunks,
                              double* out3, cudaStream_t s) {
    if (nt <= 0) return cudaSuccess;
    const int64_t per_chunk = (ns + chunks - 1) / chunks;
    dim3 grid((unsigned)((nt + 127) / 128), chunks);
    direct_partial_kernel<<<grid, 128, 0, s>>>(targets, nt, sources, ns, per_chunk, world, g_eff,
                                               soft * soft, partial);
    direct_reduce_kernel<<<(unsigned)((nt * 3 + 255) / 256), 256, 0, s>>>(partial, nt, chunks, out3);
    return cudaGetLastError();
}

}  // namespace mog
