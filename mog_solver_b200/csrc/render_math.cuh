// render_math.cuh — the reference's particle draw restated under OpenGL's
// rules for points, as __host__ __device__ functions shared by the CUDA
// renderer (render.cu) and its host twin.
//
// What is drawn (main.py:359-423, drawn by on_render, main.py:678-703):
//   vertex shader   p = (pos.xyz / world_size) * 2 - 1;
//                   gl_Position = m_proj * m_view * vec4(p, 1);
//                   gl_PointSize = 800 / (gl_Position.w + 0.1);
//                   v_speed = clamp(sqrt(length(vel.xyz)) * speed_scale, 0, 1)
//   fragment shader coord = gl_PointCoord * 2 - 1; r = dot(coord, coord);
//                   discard if r > 1; colour = getCosmicColor(v_speed),
//                   alpha = exp(-r * 3.5) * 0.8
//   state           clear (0.01, 0.01, 0.02, 0); blending SRC_ALPHA,
//                   ONE_MINUS_SRC_ALPHA on colour and alpha; no depth test.
//
// The reference never enables GL_PROGRAM_POINT_SIZE, so under the GL rules
// the shader's gl_PointSize is ignored and every point has the context's
// fixed size (1.0); point_mode 1 honours the shader's size instead.
//
// The OpenGL rules restated (GL 4.6 core, points and blending):
//  * a point is discarded unless its clip position lies in the view volume,
//    -w <= x, y, z <= w (with w > 0 here);
//  * window position (x_w, y_w) = (x/w, y/w) * (W/2, H/2) + (W/2, H/2),
//    origin at the lower left;
//  * a fragment is made for every pixel whose centre (i + 1/2, j + 1/2)
//    lies in the square of side `size` centred on (x_w, y_w); this file
//    takes the square as [x_w - size/2, x_w + size/2) on each axis (GL
//    leaves ties to the implementation);
//  * gl_PointCoord = (1/2 + (x_c - x_w) / size, 1/2 - (y_c - y_w) / size)
//    (origin upper left, the default);
//  * per pixel, fragments blend in primitive (particle index) order:
//    d' = s * a + d * (1 - a) on every channel; an 8-bit target stores
//    round(clamp(d', 0, 1) * 255) after every blend and reads back q / 255.
//
// Every float operation is a rounded IEEE operation (no contraction), and
// exp is computed here (Cody and Waite's split of ln 2, as in the Cephes
// library, then a degree-7 Taylor polynomial), so the CUDA kernels and the
// host twin produce the same bits.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define MOG_RHD __host__ __device__ __forceinline__
#else
#define MOG_RHD inline
#endif

namespace mog {
namespace rnd {

MOG_RHD float add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
MOG_RHD float sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
MOG_RHD float mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
MOG_RHD float div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
MOG_RHD float sqrt_rn(float a) {
#ifdef __CUDA_ARCH__
    return __fsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
// round to nearest, ties to even
MOG_RHD float rint_rn(float a) {
#ifdef __CUDA_ARCH__
    return rintf(a);
#else
    return std::nearbyint(a);
#endif
}
MOG_RHD float floor_f(float a) {
#ifdef __CUDA_ARCH__
    return floorf(a);
#else
    return std::floor(a);
#endif
}
MOG_RHD float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }
MOG_RHD float uint_as_float(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

// e^x for x in [-87, 88] (arguments outside are clamped; NaN gives NaN).
// x = k ln2 + f with k = rint(x / ln 2) and f = (x - k C1) - k C2, where
// C1 + C2 = ln 2 and C1 has few significant bits so that k C1 is exact;
// e^f by the Taylor series to f^7 (|f| <= 0.35: truncation below 0.1 ulp);
// then the exponent field gets k.
MOG_RHD float exp_rn(float x) {
    if (!(x == x)) return x;
    x = x < -87.0f ? -87.0f : (x > 88.0f ? 88.0f : x);
    const float k = rint_rn(mul(x, 1.44269504088896341f));
    const float f = sub(sub(x, mul(k, 0.693359375f)), mul(k, -2.12194440e-4f));
    float p = 1.0f / 5040.0f;
    p = add(mul(p, f), 1.0f / 720.0f);
    p = add(mul(p, f), 1.0f / 120.0f);
    p = add(mul(p, f), 1.0f / 24.0f);
    p = add(mul(p, f), 1.0f / 6.0f);
    p = add(mul(p, f), 0.5f);
    p = add(mul(p, f), 1.0f);
    p = add(mul(p, f), 1.0f);
    // k in [-126, 127]: 2^k is a normal float
    return mul(p, uint_as_float((uint32_t)((int)k + 127) << 23));
}

// GLSL mix(x, y, a) = x * (1 - a) + y * a
MOG_RHD float mix(float x, float y, float a) { return add(mul(x, sub(1.0f, a)), mul(y, a)); }

// getCosmicColor(t) of the fragment shader (main.py:392-405)
MOG_RHD void cosmic(float t, float& r, float& g, float& b) {
    float x0, x1, x2, y0, y1, y2, a;
    if (t < 0.3f) {
        x0 = 0.05f, x1 = 0.1f, x2 = 0.4f, y0 = 0.6f, y1 = 0.0f, y2 = 0.7f;
        a = div(t, 0.3f);
    } else if (t < 0.7f) {
        x0 = 0.6f, x1 = 0.0f, x2 = 0.7f, y0 = 1.0f, y1 = 0.4f, y2 = 0.0f;
        a = div(sub(t, 0.3f), 0.4f);
    } else {
        x0 = 1.0f, x1 = 0.4f, x2 = 0.0f, y0 = 1.0f, y1 = 0.9f, y2 = 0.7f;
        a = div(sub(t, 0.7f), 0.3f);
    }
    r = mix(x0, y0, a);
    g = mix(x1, y1, a);
    b = mix(x2, y2, a);
}

struct Params {
    float M[16];          // m_proj * m_view, column-major (element (r, c) at M[4c + r])
    float world;          // world_size uniform
    float speed_scale;    // speed_scale uniform
    float half_w, half_h; // W / 2, H / 2
    int32_t width, height;
    int32_t program_size; // 1: the shader's gl_PointSize; 0: fixed point_size
    float point_size, max_point_size;
    float clear[4];
    int32_t format;       // 0: 8-bit RGBA target, 1: float RGBA target
    int32_t tile;         // tile edge in pixels (binning only; no effect on the image)
};

// One drawn point: window position, side length and colour.
struct Splat {
    float xw, yw, size, r, g, b;
};

// GLSL mat * vec with M column-major: ((c0 x + c1 y) + c2 z) + c3 w
MOG_RHD float row_dot(const float* M, int r, float x, float y, float z, float w) {
    return add(add(add(mul(M[r], x), mul(M[4 + r], y)), mul(M[8 + r], z)), mul(M[12 + r], w));
}

// GLSL mat4 * mat4 (A * B), the same association per element.
MOG_RHD void mat_mul(const float* A, const float* B, float* out) {
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r)
            out[4 * c + r] = row_dot(A, r, B[4 * c], B[4 * c + 1], B[4 * c + 2], B[4 * c + 3]);
}

// Vertex stage, clipping, size and viewport.  false: the point is clipped.
MOG_RHD bool vertex(float px, float py, float pz, float vx, float vy, float vz, const Params& R,
                    Splat& s) {
    const float x = sub(mul(div(px, R.world), 2.0f), 1.0f);
    const float y = sub(mul(div(py, R.world), 2.0f), 1.0f);
    const float z = sub(mul(div(pz, R.world), 2.0f), 1.0f);
    const float cx = row_dot(R.M, 0, x, y, z, 1.0f);
    const float cy = row_dot(R.M, 1, x, y, z, 1.0f);
    const float cz = row_dot(R.M, 2, x, y, z, 1.0f);
    const float cw = row_dot(R.M, 3, x, y, z, 1.0f);
    const float nw = -cw;
    if (!(cw > 0.0f && cx >= nw && cx <= cw && cy >= nw && cy <= cw && cz >= nw && cz <= cw))
        return false;
    float size = R.program_size ? div(800.0f, add(cw, 0.1f)) : R.point_size;
    size = size < 1.0f ? 1.0f : (size > R.max_point_size ? R.max_point_size : size);
    s.size = size;
    s.xw = add(mul(div(cx, cw), R.half_w), R.half_w);
    s.yw = add(mul(div(cy, cw), R.half_h), R.half_h);
    const float speed = sqrt_rn(add(add(mul(vx, vx), mul(vy, vy)), mul(vz, vz)));
    cosmic(clamp01(mul(sqrt_rn(speed), R.speed_scale)), s.r, s.g, s.b);
    return true;
}

// Pixel range [i0, i1] x [j0, j1] that may hold fragments of s (one pixel
// of margin; the exact test is covers()), clipped to the image.  false if
// empty.
MOG_RHD bool pixel_range(const Splat& s, const Params& R, int& i0, int& i1, int& j0, int& j1) {
    const float h = mul(s.size, 0.5f);
    i0 = (int)floor_f(sub(s.xw, h)) - 1;
    i1 = (int)floor_f(add(s.xw, h)) + 1;
    j0 = (int)floor_f(sub(s.yw, h)) - 1;
    j1 = (int)floor_f(add(s.yw, h)) + 1;
    i0 = i0 < 0 ? 0 : i0;
    j0 = j0 < 0 ? 0 : j0;
    i1 = i1 > R.width - 1 ? R.width - 1 : i1;
    j1 = j1 > R.height - 1 ? R.height - 1 : j1;
    return i0 <= i1 && j0 <= j1;
}

// Fragment of s at pixel centre (xc, yc): false when the pixel is outside
// the point's square or the shader discards it; else its alpha.
MOG_RHD bool fragment(const Splat& s, float xc, float yc, float& alpha) {
    const float h = mul(s.size, 0.5f);
    if (!(xc >= sub(s.xw, h) && xc < add(s.xw, h) && yc >= sub(s.yw, h) && yc < add(s.yw, h)))
        return false;
    const float ps = add(0.5f, div(sub(xc, s.xw), s.size));
    const float pt = sub(0.5f, div(sub(yc, s.yw), s.size));
    const float u = sub(mul(ps, 2.0f), 1.0f);
    const float v = sub(mul(pt, 2.0f), 1.0f);
    const float r = add(mul(u, u), mul(v, v));
    if (r > 1.0f) return false;
    alpha = mul(exp_rn(mul(-r, 3.5f)), 0.8f);
    return true;
}

// SRC_ALPHA, ONE_MINUS_SRC_ALPHA
MOG_RHD float blend(float src, float dst, float a) { return add(mul(src, a), mul(dst, sub(1.0f, a))); }

MOG_RHD uint32_t to_unorm8(float x) { return (uint32_t)rint_rn(mul(clamp01(x), 255.0f)); }
MOG_RHD float from_unorm8(uint32_t q) { return div((float)q, 255.0f); }

// A pixel of the target: float channels, or 8-bit codes held as floats.
struct Pixel {
    float c[4];
};

MOG_RHD void clear_pixel(const Params& R, Pixel& p) {
    for (int k = 0; k < 4; ++k)
        p.c[k] = R.format == 0 ? (float)to_unorm8(R.clear[k]) : R.clear[k];
}

MOG_RHD void blend_pixel(const Params& R, const Splat& s, float a, Pixel& p) {
    const float src[4] = {s.r, s.g, s.b, a};
    for (int k = 0; k < 4; ++k) {
        if (R.format == 0)
            p.c[k] = (float)to_unorm8(blend(src[k], from_unorm8((uint32_t)p.c[k]), a));
        else
            p.c[k] = blend(src[k], p.c[k], a);
    }
}

}  // namespace rnd
}  // namespace mog
