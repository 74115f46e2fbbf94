// glsl_compat.hpp — enough of GLSL 4.60 for the reference's hot-path
// compute shaders and its particle vertex and fragment shaders to compile
// as C++ and run on the CPU.  TEST AND CPU-BASELINE
// INFRASTRUCTURE ONLY (oracle/_ref is the checker and the timed reference
// arm, never the product).
//
// Semantics pinned here, where GLSL leaves them to the driver:
//  * every float operation is an IEEE binary32 operation, evaluated as
//    written (the harness is built with -ffp-contract=off);
//  * mat3 * vec3 = (col0 * v.x + col1 * v.y) + col2 * v.z, component-wise;
//    mat4 * vec4 = ((col0 * v.x + col1 * v.y) + col2 * v.z) + col3 * v.w;
//    mat4 * mat4 applies the latter to each column of the right operand;
//  * mod(x, y) = x - y * floor(x / y) with IEEE division;
//  * cos / sin / acos / pow are the C library's cosf / sinf / acosf / powf;
//  * mix(x, y, a) = x * (1 - a) + y * a; fract(x) = x - floor(x);
//    clamp(x, lo, hi) = min(max(x, lo), hi);
//  * rg32f images keep two channels and read back as (r, g, 0, 1).
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <vector>

namespace glsl {

typedef unsigned int uint;

struct vec2 {
    float x, y;
    vec2() : x(0.f), y(0.f) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
};

struct vec3 {
    float x, y, z;
    vec3() : x(0.f), y(0.f), z(0.f) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3& operator*=(float s) { x = x * s; y = y * s; z = z * s; return *this; }
};

struct vec4 {
    float x, y, z, w;
    vec4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    vec4(const vec2& v, float c, float d) : x(v.x), y(v.y), z(c), w(d) {}
    vec3 xyz_() const { return vec3(x, y, z); }
    vec2 xy_() const { return vec2(x, y); }
};

struct uvec3 {
    uint x, y, z;
};

struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const vec2& v) : x((int)v.x), y((int)v.y) {}
};

struct ivec3 {
    int x, y, z;
    ivec3() : x(0), y(0), z(0) {}
    ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit ivec3(const uvec3& u) : x((int)u.x), y((int)u.y), z((int)u.z) {}
    explicit ivec3(const vec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
};
inline ivec2 operator+(const ivec2& a, const ivec2& b) { return ivec2(a.x + b.x, a.y + b.y); }
inline ivec3 operator+(const ivec3& a, const ivec3& b) { return ivec3(a.x + b.x, a.y + b.y, a.z + b.z); }

struct bvec3 {
    bool x, y, z;
};

struct mat3 {
    vec3 c[3];  // columns
    mat3(const vec3& a, const vec3& b, const vec3& d) { c[0] = a; c[1] = b; c[2] = d; }
};

struct mat4 {
    vec4 c[4];  // columns
    mat4() {}
};
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    r.x = ((m.c[0].x * v.x + m.c[1].x * v.y) + m.c[2].x * v.z) + m.c[3].x * v.w;
    r.y = ((m.c[0].y * v.x + m.c[1].y * v.y) + m.c[2].y * v.z) + m.c[3].y * v.w;
    r.z = ((m.c[0].z * v.x + m.c[1].z * v.y) + m.c[2].z * v.z) + m.c[3].z * v.w;
    r.w = ((m.c[0].w * v.x + m.c[1].w * v.y) + m.c[2].w * v.z) + m.c[3].w * v.w;
    return r;
}
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r;
    for (int j = 0; j < 4; ++j) r.c[j] = a * b.c[j];
    return r;
}

inline vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator/(const vec2& a, float s) { return vec2(a.x / s, a.y / s); }
inline vec2 operator+(const vec2& a, float s) { return vec2(a.x + s, a.y + s); }
inline vec2 operator-(const vec2& a, float s) { return vec2(a.x - s, a.y - s); }
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(const vec3& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }

inline vec3 operator*(const mat3& m, const vec3& v) {
    return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z;
}
inline mat3 transpose(const mat3& m) {
    return mat3(vec3(m.c[0].x, m.c[1].x, m.c[2].x), vec3(m.c[0].y, m.c[1].y, m.c[2].y),
                vec3(m.c[0].z, m.c[1].z, m.c[2].z));
}

inline float floor(float x) { return std::floor(x); }
inline vec2 floor(const vec2& v) { return vec2(floor(v.x), floor(v.y)); }
inline vec3 floor(const vec3& v) { return vec3(floor(v.x), floor(v.y), floor(v.z)); }
inline float fract(float x) { return x - floor(x); }
inline vec2 fract(const vec2& v) { return vec2(fract(v.x), fract(v.y)); }
inline vec3 fract(const vec3& v) { return vec3(fract(v.x), fract(v.y), fract(v.z)); }
inline float dot(const vec3& a, const vec3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float acos(float x) { return std::acos(x); }
inline float pow(float x, float y) { return std::pow(x, y); }
inline float clamp(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline vec3 mix(const vec3& x, const vec3& y, float a) {
    return vec3(mix(x.x, y.x, a), mix(x.y, y.y, a), mix(x.z, y.z, a));
}
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float cos(float x) { return std::cos(x); }
inline float sin(float x) { return std::sin(x); }
inline float exp(float x) { return std::exp(x); }
inline float log2(float x) { return std::log2(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float mod(float x, float y) { return x - y * floor(x / y); }
inline vec3 mod(const vec3& v, float y) { return vec3(mod(v.x, y), mod(v.y, y), mod(v.z, y)); }
inline float length(const vec3& v) { return sqrt((v.x * v.x + v.y * v.y) + v.z * v.z); }
inline bvec3 greaterThanEqual(const ivec3& a, const ivec3& b) {
    return bvec3{a.x >= b.x, a.y >= b.y, a.z >= b.z};
}
inline bool any(const bvec3& b) { return b.x || b.y || b.z; }

inline uint atomicAdd(uint& mem, uint v) {
    return std::atomic_ref<uint>(mem).fetch_add(v, std::memory_order_relaxed);
}

// std430 runtime-sized array
template <typename T>
struct SSBO {
    T* data = nullptr;
    int n = 0;
    T& operator[](int i) { return data[i]; }
    T& operator[](uint i) { return data[i]; }
    int length() const { return n; }
};

// image3D with 2 (rg32f) or 4 (rgba32f) float channels
struct image3D {
    std::vector<float> texels;
    int sx = 0, sy = 0, sz = 0, ch = 4;
    void allocate(int x, int y, int z, int channels) {
        sx = x; sy = y; sz = z; ch = channels;
        texels.assign((size_t)x * y * z * channels, 0.f);
    }
    size_t at(const ivec3& p) const { return (((size_t)p.z * sy + p.y) * sx + p.x) * ch; }
};

inline vec4 imageLoad(const image3D& img, const ivec3& p) {
    const float* t = &img.texels[img.at(p)];
    return img.ch == 2 ? vec4(t[0], t[1], 0.f, 1.f) : vec4(t[0], t[1], t[2], t[3]);
}
inline void imageStore(image3D& img, const ivec3& p, const vec4& v) {
    float* t = &img.texels[img.at(p)];
    t[0] = v.x;
    t[1] = v.y;
    if (img.ch == 4) {
        t[2] = v.z;
        t[3] = v.w;
    }
}
inline ivec3 imageSize(const image3D& img) { return ivec3(img.sx, img.sy, img.sz); }

// An image uniform: which texture is bound to the unit (bind_to_image).
struct image3D_ref {
    image3D* p = nullptr;
};
inline vec4 imageLoad(const image3D_ref& r, const ivec3& q) { return imageLoad(*r.p, q); }
inline void imageStore(const image3D_ref& r, const ivec3& q, const vec4& v) { imageStore(*r.p, q, v); }
inline ivec3 imageSize(const image3D_ref& r) { return imageSize(*r.p); }

// The invocation currently executing on this host thread.
extern thread_local uvec3 gl_GlobalInvocationID;

}  // namespace glsl
