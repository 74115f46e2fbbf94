// ic_sampler.cuh — the reference's initial-condition sampler
// (init_particles.glsl, DIM 3, as init_particles_gpu runs it, main.py:283-310):
// every particle draws candidates from an integer hash, keeps the first one
// whose threshold falls under a 4-octave Perlin fBm density, and gets a
// uniform random velocity.  One implementation for the GPU kernel and for
// the host entry point: every float operation is spelled out as a rounded
// IEEE operation, so both evaluate the same expression tree as the shader
// (no contraction into FMAs); only cos, sin, acos and pow come from the
// respective math library.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define MOG_HD __host__ __device__ __forceinline__
#else
#define MOG_HD inline
#endif

namespace mog {
namespace ic {

MOG_HD float add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
MOG_HD float sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
MOG_HD float mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
MOG_HD float div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
MOG_HD float fcos(float x) {
#ifdef __CUDA_ARCH__
    return cosf(x);
#else
    return std::cos(x);
#endif
}
MOG_HD float fsin(float x) {
#ifdef __CUDA_ARCH__
    return sinf(x);
#else
    return std::sin(x);
#endif
}
MOG_HD float facos(float x) {
#ifdef __CUDA_ARCH__
    return acosf(x);
#else
    return std::acos(x);
#endif
}
MOG_HD float fpow(float x, float y) {
#ifdef __CUDA_ARCH__
    return powf(x, y);
#else
    return std::pow(x, y);
#endif
}
MOG_HD float ffloor(float x) {
#ifdef __CUDA_ARCH__
    return floorf(x);
#else
    return std::floor(x);
#endif
}

struct V3 {
    float x, y, z;
};

// The shader's integer hash (a 32-bit finaliser) and its combinations.
MOG_HD uint32_t hash(uint32_t x) {
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}
MOG_HD uint32_t hash2(uint32_t x, uint32_t y) {
    return hash(x ^ (hash(y) + 0x9e3779b9u + (x << 6) + (x >> 2)));
}
MOG_HD uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {
    return hash(hash2(x, y) ^ (hash(z) + 0x9e3779b9u));
}
// float(hash) / 4294967295.0 (the literal rounds to 2^32 in binary32)
MOG_HD float rnd(uint32_t s) { return div((float)hash(s), 4294967295.0f); }
MOG_HD V3 rnd3(uint32_t s) { return {rnd(s), rnd(hash(s)), rnd(hash(hash(s)))}; }

MOG_HD float dot(const V3& a, const V3& b) {
    return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z));
}
MOG_HD float mix(float x, float y, float a) { return add(mul(x, sub(1.0f, a)), mul(y, a)); }
MOG_HD float fade(float t) {
    return mul(mul(mul(t, t), t), add(mul(t, sub(mul(t, 6.0f), 15.0f)), 10.0f));
}

// Unit gradient of lattice point (x, y, z) for noise seed s.
MOG_HD V3 grad3(int x, int y, int z, uint32_t s) {
    const uint32_t h = hash3((uint32_t)x + s, (uint32_t)y + s * 7u, (uint32_t)z + s * 13u);
    const float theta = div(mul((float)(h & 0xFFFFu), 6.28318530718f), 65535.0f);
    const float phi = facos(sub(div(mul(2.0f, (float)(h >> 16)), 65535.0f), 1.0f));
    const float sp = fsin(phi);
    return {mul(sp, fcos(theta)), mul(sp, fsin(theta)), fcos(phi)};
}

MOG_HD float perlin3(const V3& p, uint32_t s) {
    const float flx = ffloor(p.x), fly = ffloor(p.y), flz = ffloor(p.z);
    const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
    const V3 f = {sub(p.x, flx), sub(p.y, fly), sub(p.z, flz)};
    const float ux = fade(f.x), uy = fade(f.y), uz = fade(f.z);
    auto corner = [&](int dx, int dy, int dz) {
        const V3 g = grad3(ix + dx, iy + dy, iz + dz, s);
        const V3 d = {sub(f.x, (float)dx), sub(f.y, (float)dy), sub(f.z, (float)dz)};
        return dot(g, d);
    };
    const float n000 = corner(0, 0, 0), n100 = corner(1, 0, 0), n010 = corner(0, 1, 0),
                n110 = corner(1, 1, 0), n001 = corner(0, 0, 1), n101 = corner(1, 0, 1),
                n011 = corner(0, 1, 1), n111 = corner(1, 1, 1);
    const float nx00 = mix(n000, n100, ux), nx10 = mix(n010, n110, ux);
    const float nx01 = mix(n001, n101, ux), nx11 = mix(n011, n111, ux);
    const float nxy0 = mix(nx00, nx10, uy), nxy1 = mix(nx01, nx11, uy);
    return mix(nxy0, nxy1, uz);
}

// Fractal sum of 4 octaves, amplitude 1/2^(i+1), frequency 2^i.
MOG_HD float fbm3(const V3& p, uint32_t s) {
    float value = 0.0f, amplitude = 0.5f, frequency = 1.0f;
    for (int i = 0; i < 4; ++i) {
        const V3 q = {mul(p.x, frequency), mul(p.y, frequency), mul(p.z, frequency)};
        value = add(value, mul(amplitude, perlin3(q, s + (uint32_t)i * 1000u)));
        amplitude = mul(amplitude, 0.5f);
        frequency = mul(frequency, 2.0f);
    }
    return value;
}

struct Params {
    float world, noise_scale, contrast, mass, spawn_buffer;
    uint32_t seed, shape;  // shape 0: cube, 1: sphere
};

// Particle id's position and velocity records (x, y, z, m) and (vx, vy, vz, 0).
MOG_HD void sample(uint32_t id, const Params& P, float (&pos)[4], float (&vel)[4]) {
    const uint32_t ps = P.seed + id * 12345u;
    const float min_b = mul(P.spawn_buffer, P.world);
    const float max_b = mul(sub(1.0f, P.spawn_buffer), P.world);
    const float range = sub(max_b, min_b);
    const float centre = mul(P.world, 0.5f);
    const float radius = mul(range, 0.5f);
    V3 out = {0.f, 0.f, 0.f};
    uint32_t attempts = 0;
    for (; attempts < 64u; ++attempts) {
        V3 c;
        if (P.shape == 1u) {
            V3 sp;
            uint32_t tries = 0;
            do {
                const V3 r = rnd3(ps + attempts * 1000u + tries * 100u);
                sp = {sub(mul(r.x, 2.0f), 1.0f), sub(mul(r.y, 2.0f), 1.0f), sub(mul(r.z, 2.0f), 1.0f)};
                ++tries;
            } while (dot(sp, sp) > 1.0f && tries < 16u);
            c = {add(centre, mul(sp.x, radius)), add(centre, mul(sp.y, radius)),
                 add(centre, mul(sp.z, radius))};
        } else {
            const V3 r = rnd3(ps + attempts * 1000u);
            c = {add(mul(r.x, range), min_b), add(mul(r.y, range), min_b), add(mul(r.z, range), min_b)};
        }
        const V3 nc = {div(mul(c.x, P.noise_scale), P.world), div(mul(c.y, P.noise_scale), P.world),
                       div(mul(c.z, P.noise_scale), P.world)};
        float d = add(fbm3(nc, P.seed), 0.5f);
        d = d < 0.0f ? 0.0f : (d > 1.0f ? 1.0f : d);  // clamp(d, 0, 1)
        d = fpow(d, P.contrast);
        if (rnd(ps + attempts * 1000u + 500u) < d) {
            out = c;
            break;
        }
    }
    if (attempts >= 64u) {
        if (P.shape == 1u) {
            const float r = mul(fpow(rnd(ps), div(1.0f, 3.0f)), radius);
            const float theta = mul(rnd(hash(ps)), 6.28318530718f);
            const float phi = facos(sub(mul(2.0f, rnd(hash(hash(ps)))), 1.0f));
            const float sp = fsin(phi);
            out = {add(centre, mul(mul(sp, fcos(theta)), r)), add(centre, mul(mul(sp, fsin(theta)), r)),
                   add(centre, mul(fcos(phi), r))};
        } else {
            const V3 r = rnd3(ps);
            out = {add(mul(r.x, range), min_b), add(mul(r.y, range), min_b), add(mul(r.z, range), min_b)};
        }
    }
    const V3 rv = rnd3(ps + 999u);
    pos[0] = out.x;
    pos[1] = out.y;
    pos[2] = out.z;
    pos[3] = P.mass;
    vel[0] = mul(mul(sub(rv.x, 0.5f), 1.0f), P.world);
    vel[1] = mul(mul(sub(rv.y, 0.5f), 1.0f), P.world);
    vel[2] = mul(mul(sub(rv.z, 0.5f), 1.0f), P.world);
    vel[3] = 0.0f;
}

}  // namespace ic
}  // namespace mog
