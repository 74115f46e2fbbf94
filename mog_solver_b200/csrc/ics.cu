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

// ---------------------------------------------------------------------------
// The reference's two-galaxy initialiser (Simulation.init_particles2,
// main.py:312-357) as a CUDA kernel.  The reference draws with NumPy's
// global legacy generator, a sequential Mersenne Twister that a GPU thread
// cannot reproduce per particle, so here every particle takes its three
// uniforms from a counter-based generator instead (the SplitMix64
// finaliser of Steele, Lea and Flood, 2014, applied to a seed-derived key
// plus a per-draw counter), and then follows the reference's formulas in
// FP64, as NumPy evaluates them, rounding to FP32 on the store:
//   r = -ln(1 - u0) * 0.08 L, theta = 2 pi u1, phi = acos(2 u2 - 1),
//   pos = L/2 + offset_b L + r (sin phi cos theta, sin phi sin theta, cos phi),
//   vel = 0.3 sqrt(r / L + 0.01) (a_b x d) / (|a_b x d| + 1e-10) + bulk_b
// with galaxy b = 0 for the first n/2 particles and 1 for the next n/2
// (offset -0.2 / +0.2 L along x, bulk (0.3, 0.1, 0) / (-0.3, -0.1, 0), spin
// axis (0.3, 0.7, 0.5) / (-0.5, 0.2, 0.8) normalised).  With odd n the last
// record is zero, as in the reference.
namespace mog {
namespace galaxies {

__host__ __device__ inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) from the top 53 bits: draw j of particle i.
__host__ __device__ inline double uniform(uint64_t key, uint64_t i, int j) {
    return (double)(splitmix64(key + (i << 2) + (uint64_t)j) >> 11) * 0x1.0p-53;
}

__host__ __device__ inline void sample(uint64_t key, int64_t i, int64_t per, double world,
                                       float mass, float* p, float* v) {
    if (i >= 2 * per) {
        for (int a = 0; a < 4; ++a) p[a] = v[a] = 0.f;
        return;
    }
    const int b = i >= per ? 1 : 0;
    const double pi = 3.141592653589793;
    const double u0 = uniform(key, (uint64_t)i, 0), u1 = uniform(key, (uint64_t)i, 1),
                 u2 = uniform(key, (uint64_t)i, 2);
    const double r = -log(1.0 - u0) * 0.08 * world;
    const double theta = 2.0 * pi * u1;
    const double phi = acos(-1.0 + 2.0 * u2);
    const double x = r * sin(phi) * cos(theta);
    const double y = r * sin(phi) * sin(theta);
    const double z = r * cos(phi);
    const double centre = world / 2.0;
    const double off_x = b ? 0.2 : -0.2;
    p[0] = (float)(centre + off_x * world + x);
    p[1] = (float)(centre + 0.0 * world + y);
    p[2] = (float)(centre + 0.0 * world + z);
    p[3] = mass;
    double ax = b ? -0.5 : 0.3, ay = b ? 0.2 : 0.7, az = b ? 0.8 : 0.5;
    const double an = sqrt(ax * ax + ay * ay + az * az);
    ax /= an;
    ay /= an;
    az /= an;
    const double v_circ = 0.3 * sqrt(r / world + 0.01);
    const double dx = ay * z - az * y, dy = az * x - ax * z, dz = ax * y - ay * x;
    const double dn = sqrt(dx * dx + dy * dy + dz * dz) + 1e-10;
    v[0] = (float)(v_circ * (dx / dn) + (b ? -0.3 : 0.3));
    v[1] = (float)(v_circ * (dy / dn) + (b ? -0.1 : 0.1));
    v[2] = (float)(v_circ * (dz / dn) + 0.0);
    v[3] = 0.f;
}

__global__ void __launch_bounds__(256) two_galaxies_kernel(float4* __restrict__ pos,
                                                           float4* __restrict__ vel, int64_t n,
                                                           double world, float mass, uint64_t key) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[4], v[4];
    sample(key, i, n / 2, world, mass, p, v);
    pos[i] = make_float4(p[0], p[1], p[2], p[3]);
    vel[i] = make_float4(v[0], v[1], v[2], v[3]);
}

inline bool args_ok(int64_t n, float world, float mass) {
    return n >= 0 && std::isfinite(world) && world > 0.f && std::isfinite(mass);
}

}  // namespace galaxies
}  // namespace mog

extern "C" {

int mog_init_two_galaxies(float* pos4, float* vel4, int64_t n, float world, float mass,
                          uint64_t seed, void* stream) {
    if (!mog::galaxies::args_ok(n, world, mass)) return MOG_ERR_ARG;
    if (n == 0) return MOG_OK;
    if (!pos4 || !vel4) return MOG_ERR_ARG;
    const uint64_t key = mog::galaxies::splitmix64(seed);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    mog::galaxies::two_galaxies_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4), n, (double)world, mass,
        key);
    return cudaGetLastError() == cudaSuccess ? MOG_OK : MOG_ERR_CUDA;
}

int mog_init_two_galaxies_host(float* pos4, float* vel4, int64_t n, float world, float mass,
                               uint64_t seed) {
    if (!mog::galaxies::args_ok(n, world, mass)) return MOG_ERR_ARG;
    if (n > 0 && (!pos4 || !vel4)) return MOG_ERR_ARG;
    const uint64_t key = mog::galaxies::splitmix64(seed);
    for (int64_t i = 0; i < n; ++i)
        mog::galaxies::sample(key, i, n / 2, (double)world, mass, pos4 + 4 * i, vel4 + 4 * i);
    return MOG_OK;
}

}  // extern "C"
