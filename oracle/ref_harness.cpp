// ref_harness.cpp — runs the reference's GLSL compute shaders (translated
// to C++ by ref_build.py into _ref/gen/*.inc) on the CPU, dispatch by
// dispatch, exactly in the order and with the bindings and uniforms of
// Simulation.step_fft (main.py:592-669) and run_fft_3d_batched
// (main.py:564-590), including its texture ping-pong.  TEST AND CPU-BASELINE
// INFRASTRUCTURE ONLY.  Invocations of one dispatch run in parallel with
// OpenMP (they are independent except for the atomics of mass.glsl); each
// dispatch completes before the next starts (the memory_barrier calls).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "glsl_compat.hpp"
#include "mass.inc"
#include "complex.inc"
#include "fft_batched.inc"
#include "fourier.inc"
#include "greens.inc"
#include "pack.inc"
#include "update.inc"
#include "init_particles.inc"
#include "point_vs.inc"
#include "point_fs.inc"

namespace glsl {
thread_local uvec3 gl_GlobalInvocationID;
}

using namespace glsl;

namespace {

static_assert(sizeof(vec4) == 16, "vec4 must alias a float4 record");

template <class F>
void dispatch(int gx, int gy, int gz, int lx, int ly, int lz, F fn) {
    const long X = (long)gx * lx, Y = (long)gy * ly, Z = (long)gz * lz;
    const long total = X * Y * Z;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < total; ++i) {
        gl_GlobalInvocationID = uvec3{(uint)(i % X), (uint)((i / X) % Y), (uint)(i / (X * Y))};
        fn();
    }
}

struct Textures {
    int k = -1, g = -1;
    image3D ca, cb, gx, gy, gz, grad;
    void ensure(int kk, int gg) {
        if (kk == k && gg == g) return;
        k = kk;
        g = gg;
        for (image3D* t : {&ca, &cb, &gx, &gy, &gz}) t->allocate(g, g, g * k, 2);
        grad.allocate(g, g, g * k, 4);
    }
};
Textures T;

int grid_dispatch(int g) { return std::max(1, g / 8); }

// run_fft_3d_batched: 3 axes x (log2 g + 1) passes, swapping textures
// after every pass; returns the texture written last.
image3D* run_fft(image3D* src, image3D* dst, bool forward, int gs, int ng) {
    namespace S = fft_batched_glsl;
    const int num_stages = (int)std::log2((double)gs);
    S::direction = forward ? 1 : -1;
    S::gridSize = gs;
    S::nGrids = ng;
    image3D* cs = src;
    image3D* cd = dst;
    for (int axis = 0; axis < 3; ++axis) {
        S::axis = axis;
        for (int stage = 0; stage < num_stages + 1; ++stage) {
            S::stage = stage;
            S::inputTexture.p = cs;
            S::outputTexture.p = cd;
            dispatch(grid_dispatch(gs), grid_dispatch(gs), ng, 8, 8, 1, [] { S::main(); });
            std::swap(cs, cd);
        }
    }
    return cs;
}

void do_mass(float* pos4, int n, const float* off4, const float* rot12, int k, int g,
             float world, float voxel, uint* mass) {
    namespace S = mass_glsl;
    const int cells = k * g * g * g;
    std::memset(mass, 0, sizeof(uint) * cells);  // clear_mass (main.py:558-562)
    S::positions.data = reinterpret_cast<vec4*>(pos4);
    S::positions.n = n;
    S::mass_grid.data = mass;
    S::mass_grid.n = cells;
    S::offsets.data = reinterpret_cast<vec4*>(const_cast<float*>(off4));
    S::offsets.n = k;
    S::rotations.data = reinterpret_cast<vec4*>(const_cast<float*>(rot12));
    S::rotations.n = 3 * k;
    S::gridSize = g;
    S::nGrids = k;
    S::voxelSize = voxel;
    S::worldSize = world;
    dispatch((n + 255) / 256, 1, 1, 256, 1, 1, [] { S::main(); });
}

void do_solve(uint* mass, int k, int g, float world, float Gc) {
    const int cells = k * g * g * g;
    T.ensure(k, g);
    const int d = grid_dispatch(g);
    {
        namespace S = complex_glsl;
        S::mass_grid.data = mass;
        S::mass_grid.n = cells;
        S::complexTexture.p = &T.ca;
        S::gridSize = g;
        S::nGrids = k;
        dispatch(d, d, g * k, 8, 8, 1, [] { S::main(); });
    }
    image3D* spec = run_fft(&T.ca, &T.cb, true, g, k);
    {
        namespace S = fourier_glsl;
        S::spectrumTex.p = spec;
        S::gridSize = g;
        S::nGrids = k;
        dispatch(d, d, g * k, 8, 8, 1, [] { S::main(); });
    }
    {
        namespace S = greens_glsl;
        S::inputTexture.p = spec;
        S::outGradX.p = &T.gx;
        S::outGradY.p = &T.gy;
        S::outGradZ.p = &T.gz;
        S::gridSize = g;
        S::nGrids = k;
        S::G = Gc;
        S::worldSize = world;
        dispatch(d, d, g * k, 8, 8, 1, [] { S::main(); });
    }
    image3D* rx = run_fft(&T.gx, &T.cb, false, g, k);
    image3D* ry = run_fft(&T.gy, &T.ca, false, g, k);
    image3D* rz = run_fft(&T.gz, &T.cb, false, g, k);
    {
        namespace S = pack_glsl;
        S::realGradX.p = rx;
        S::realGradY.p = ry;
        S::realGradZ.p = rz;
        S::finalForce.p = &T.grad;
        S::gridSize = g;
        S::nGrids = k;
        dispatch(d, d, g * k, 8, 8, 1, [] { S::main(); });
    }
}

void do_update(float* pos4, float* vel4, int n, const float* off4, const float* rot12, int k,
               int g, float world, float voxel, float dt, float damping) {
    namespace S = update_glsl;
    S::positions.data = reinterpret_cast<vec4*>(pos4);
    S::positions.n = n;
    S::velocities.data = reinterpret_cast<vec4*>(vel4);
    S::velocities.n = n;
    S::offsets.data = reinterpret_cast<vec4*>(const_cast<float*>(off4));
    S::offsets.n = k;
    S::rotations.data = reinterpret_cast<vec4*>(const_cast<float*>(rot12));
    S::rotations.n = 3 * k;
    S::gradientTexture.p = &T.grad;
    S::deltaTime = dt;
    S::gridSize = g;
    S::nGrids = k;
    S::worldSize = world;
    S::voxelSize = voxel;
    S::damping = damping;
    dispatch((n + 255) / 256, 1, 1, 256, 1, 1, [] { S::main(); });
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) int ref_threads(int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
}

// mass.glsl into mass_out (k g^3 uint32).
__attribute__((visibility("default"))) void ref_deposit(float* pos4, int n, const float* off4,
                                                        const float* rot12, int k, int g,
                                                        float world, float voxel,
                                                        uint32_t* mass_out) {
    do_mass(pos4, n, off4, rot12, k, g, world, voxel, mass_out);
}

// complex .. pack from a uint32 mass grid; grad_out: k g^3 x 4 floats
// (the gradient texture, [z][y][x] with z = grid * g + local z).
__attribute__((visibility("default"))) void ref_solve(uint32_t* mass, int k, int g, float world,
                                                      float Gc, float* grad_out) {
    do_solve(mass, k, g, world, Gc);
    std::memcpy(grad_out, T.grad.texels.data(), sizeof(float) * T.grad.texels.size());
}

// update.glsl from a caller gradient texture.
__attribute__((visibility("default"))) void ref_update(float* pos4, float* vel4, int n,
                                                       const float* off4, const float* rot12,
                                                       int k, int g, float world, float voxel,
                                                       float dt, float damping,
                                                       const float* grad_in) {
    T.ensure(k, g);
    std::memcpy(T.grad.texels.data(), grad_in, sizeof(float) * T.grad.texels.size());
    do_update(pos4, vel4, n, off4, rot12, k, g, world, voxel, dt, damping);
}

// One whole step_fft.  mass_scratch: k g^3 uint32 (contents on return:
// this step's mass grid).
__attribute__((visibility("default"))) void ref_step(float* pos4, float* vel4, int n,
                                                     const float* off4, const float* rot12, int k,
                                                     int g, float world, float voxel, float Gc,
                                                     float dt, float damping,
                                                     uint32_t* mass_scratch) {
    do_mass(pos4, n, off4, rot12, k, g, world, voxel, mass_scratch);
    do_solve(mass_scratch, k, g, world, Gc);
    do_update(pos4, vel4, n, off4, rot12, k, g, world, voxel, dt, damping);
}

// init_particles.glsl as init_particles_gpu (main.py:283-310) dispatches
// it: numParticles, worldSize, noiseScale, densityContrast, seed, baseMass,
// spawnBuffer, spawnShape as given; (n + 255) / 256 groups of 256.
__attribute__((visibility("default"))) void ref_init_particles(float* pos4, float* vel4, int n,
                                                               float world, float noise_scale,
                                                               float contrast, uint32_t seed,
                                                               float mass, float spawn_buffer,
                                                               uint32_t shape) {
    namespace S = init_particles_glsl;
    S::numParticles = (uint)n;
    S::worldSize = world;
    S::noiseScale = noise_scale;
    S::densityContrast = contrast;
    S::seed = seed;
    S::baseMass = mass;
    S::spawnBuffer = spawn_buffer;
    S::spawnShape = shape;
    S::positions.data = reinterpret_cast<vec4*>(pos4);
    S::positions.n = n;
    S::velocities.data = reinterpret_cast<vec4*>(vel4);
    S::velocities.n = n;
    dispatch((n + 255) / 256, 1, 1, 256, 1, 1, [] { S::main(); });
}

// The particle vertex shader of render_prog (main.py:360-383) on n vertices,
// with the uniforms on_render sets (m_view, m_proj as the column-major bytes
// it writes).  out: n x 6 = gl_Position (4), gl_PointSize, v_speed.
// Serial: the shader's inputs and outputs are namespace variables.
__attribute__((visibility("default"))) void ref_point_vertex(const float* pos4, const float* vel4,
                                                             int n, float world,
                                                             float speed_scale,
                                                             const float* m_view,
                                                             const float* m_proj, float* out) {
    namespace S = point_vs_glsl;
    S::world_size = world;
    S::speed_scale = speed_scale;
    for (int c = 0; c < 4; ++c) {
        S::m_view.c[c] = vec4(m_view[4 * c], m_view[4 * c + 1], m_view[4 * c + 2], m_view[4 * c + 3]);
        S::m_proj.c[c] = vec4(m_proj[4 * c], m_proj[4 * c + 1], m_proj[4 * c + 2], m_proj[4 * c + 3]);
    }
    for (int i = 0; i < n; ++i) {
        S::in_pos = vec4(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], pos4[4 * i + 3]);
        S::in_vel = vec4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], vel4[4 * i + 3]);
        S::main();
        float* o = out + 6 * (size_t)i;
        o[0] = S::gl_Position.x;
        o[1] = S::gl_Position.y;
        o[2] = S::gl_Position.z;
        o[3] = S::gl_Position.w;
        o[4] = S::gl_PointSize;
        o[5] = S::v_speed;
    }
}

// The particle fragment shader (main.py:385-410) on m fragments given
// gl_PointCoord (m x 2) and v_speed (m).  out: m x 5 = fragColor (4) and 1
// where the shader kept the fragment, 0 where it discarded it.
__attribute__((visibility("default"))) void ref_point_fragment(const float* point_coord,
                                                               const float* v_speed, int m,
                                                               float* out) {
    namespace S = point_fs_glsl;
    for (int i = 0; i < m; ++i) {
        S::gl_PointCoord = vec2(point_coord[2 * i], point_coord[2 * i + 1]);
        S::v_speed = v_speed[i];
        S::discarded = false;
        S::fragColor = vec4();
        S::main();
        float* o = out + 5 * (size_t)i;
        o[0] = S::fragColor.x;
        o[1] = S::fragColor.y;
        o[2] = S::fragColor.z;
        o[3] = S::fragColor.w;
        o[4] = S::discarded ? 0.f : 1.f;
    }
}

}  // extern "C"
