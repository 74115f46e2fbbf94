// ics.cu — the reference's GPU initial-condition sampler as a CUDA kernel
// (init_particles.glsl, DIM 3, dispatched by init_particles_gpu,
// main.py:283-310), plus the same code on the host for machines without a
// GPU.  One thread per particle; see ic_sampler.cuh.
#include <algorithm>
#include <cmath>

#include "../../include/mog.h"
#include "ic_sampler.cuh"
#include "mog_internal.h"

namespace mog {
namespace {

__global__ void __launch_bounds__(256) init_particles_kernel(float4* __restrict__ pos,
                                                             float4* __restrict__ vel, int64_t n,
                                                             ic::Params P) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[4], v[4];
    ic::sample((uint32_t)i, P, p, v);
    pos[i] = make_float4(p[0], p[1], p[2], p[3]);
    vel[i] = make_float4(v[0], v[1], v[2], v[3]);
}

bool params_ok(int64_t n, float world, float noise_scale, float contrast, float mass,
               float spawn_buffer, int32_t shape) {
    return n >= 0 && n <= 0xFFFFFFFFll && std::isfinite(world) && world > 0.f &&
           std::isfinite(noise_scale) && std::isfinite(contrast) && std::isfinite(mass) &&
           std::isfinite(spawn_buffer) && (shape == 0 || shape == 1);
}

}  // namespace
}  // namespace mog

extern "C" {

int mog_init_particles(float* pos4, float* vel4, int64_t n, float world, float noise_scale,
                       float contrast, uint32_t seed, float mass, float spawn_buffer,
                       int32_t shape, void* stream) {
    if (!mog::params_ok(n, world, noise_scale, contrast, mass, spawn_buffer, shape))
        return MOG_ERR_ARG;
    if (n == 0) return MOG_OK;
    if (!pos4 || !vel4) return MOG_ERR_ARG;
    const mog::ic::Params P{world, noise_scale, contrast, mass, spawn_buffer, seed, (uint32_t)shape};
    const unsigned blocks = (unsigned)((n + 255) / 256);
    mog::init_particles_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4), n, P);
    return cudaGetLastError() == cudaSuccess ? MOG_OK : MOG_ERR_CUDA;
}

int mog_init_particles_host(float* pos4, float* vel4, int64_t n, float world, float noise_scale,
                            float contrast, uint32_t seed, float mass, float spawn_buffer,
                            int32_t shape) {
    if (!mog::params_ok(n, world, noise_scale, contrast, mass, spawn_buffer, shape))
        return MOG_ERR_ARG;
    if (n > 0 && (!pos4 || !vel4)) return MOG_ERR_ARG;
    const mog::ic::Params P{world, noise_scale, contrast, mass, spawn_buffer, seed, (uint32_t)shape};
    for (int64_t i = 0; i < n; ++i) {
        float p[4], v[4];
        mog::ic::sample((uint32_t)i, P, p, v);
        std::copy(p, p + 4, pos4 + 4 * i);
        std::copy(v, v + 4, vel4 + 4 * i);
    }
    return MOG_OK;
}

}  // extern "C"
