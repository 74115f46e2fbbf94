/*
 * mog_oracle.c — CPU restatement of the reference's deposit and update
 * shaders, used ONLY as test infrastructure (the checker of the CUDA path
 * in tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg).
 * Nothing in the product links or calls this file.
 *
 * Compiled with -O2 -ffp-contract=off (no FMA contraction, IEEE float
 * evaluation) so every operation below rounds exactly as written.  It
 * follows:
 *   mass.glsl:38-55   deposit: centre, rotate (GLSL mat3 * vec3), un-centre,
 *                     subtract offset, double mod, int() / voxel, % g,
 *                     atomicAdd of uint(m * 1000.0)
 *   update.glsl:67-89 gather, transpose(rot) * F, sum over grids in index
 *                     order, / k, damped leapfrog, mod(pos, L)
 * in two index modes:
 *   EXACT  the shader's own op sequence (as above);
 *   FAST   t_r = fma(a_r2, c.z, fma(a_r1, c.y, fma(a_r0, c.x, b_r))),
 *          cell_r = floor(t_r) mod g, with a_rj = M[j][r] / h and
 *          b_r = (L/2 - off_r) / h rounded from double (the same rows the
 *          library builds in mog_create).
 * and two fixed-point mass modes (u64 scale 2^bits; u32 x 1000).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

static float glsl_mod(float x, float y) { return x - y * floorf(x / y); }

/* (k x 12) FAST rows from the packed rotations/offsets. */
ORACLE_API void oracle_fast_rows(const float* rot12, const float* off4, int k, float world,
                                 int g, float* out12) {
    const float voxel = (float)((double)world / (double)g);
    const double hv = (double)voxel;
    const double half_l = (double)(world * 0.5f);
    for (int i = 0; i < k; ++i) {
        const float* R = rot12 + 12 * i;
        float* o = out12 + 12 * i;
        for (int r = 0; r < 3; ++r) {
            for (int j = 0; j < 3; ++j) o[4 * r + j] = (float)((double)R[4 * j + r] / hv);
            o[4 * r + 3] = (float)((half_l - (double)off4[4 * i + r]) / hv);
        }
    }
}

static uint32_t cell_fast(const float* rows, float cx, float cy, float cz, int lg) {
    const int mask = (1 << lg) - 1;
    float t[3];
    for (int r = 0; r < 3; ++r) {
        const float* a = rows + 4 * r;
        t[r] = fmaf(a[2], cz, fmaf(a[1], cy, fmaf(a[0], cx, a[3])));
    }
    const uint32_t ix = (uint32_t)((int)floorf(t[0]) & mask);
    const uint32_t iy = (uint32_t)((int)floorf(t[1]) & mask);
    const uint32_t iz = (uint32_t)((int)floorf(t[2]) & mask);
    return ix | (iy << lg) | (iz << (2 * lg));
}

static int exact_axis(float rot, float off, float half_l, float world, float voxel, int g) {
    float l = (rot + half_l) - off;                               /* mass.glsl:44 */
    l = glsl_mod(glsl_mod(l, world) + world, world);              /* mass.glsl:46 */
    return ((int)(l / voxel)) % g;                                /* mass.glsl:48 */
}

static uint32_t cell_exact(const float* R, const float* off, float cx, float cy, float cz,
                           float half_l, float world, float voxel, int lg) {
    const int g = 1 << lg;
    /* GLSL mat3(col0, col1, col2) * c with col_j = R[4j..4j+2] */
    const float rx = (R[0] * cx + R[4] * cy) + R[8] * cz;
    const float ry = (R[1] * cx + R[5] * cy) + R[9] * cz;
    const float rz = (R[2] * cx + R[6] * cy) + R[10] * cz;
    const int x = exact_axis(rx, off[0], half_l, world, voxel, g);
    const int y = exact_axis(ry, off[1], half_l, world, voxel, g);
    const int z = exact_axis(rz, off[2], half_l, world, voxel, g);
    return (uint32_t)x | ((uint32_t)y << lg) | ((uint32_t)z << (2 * lg));
}

/* Cell of particle (cx, cy, cz already centred) in grid i. */
static uint32_t cell_of(int index_mode, const float* rot12, const float* off4,
                        const float* fast12, int i, float cx, float cy, float cz, float half_l,
                        float world, float voxel, int lg) {
    if (index_mode == 0) return cell_fast(fast12 + 12 * i, cx, cy, cz, lg);
    return cell_exact(rot12 + 12 * i, off4 + 4 * i, cx, cy, cz, half_l, world, voxel, lg);
}

/* cells[p * k + i] for every particle and grid. */
ORACLE_API void oracle_cells(const float* pos4, int64_t n, const float* rot12, const float* off4,
                             int k, int g, float world, int index_mode, uint32_t* cells) {
    int lg = 0;
    while ((1 << lg) < g) ++lg;
    const float voxel = (float)((double)world / (double)g);
    const float half_l = world * 0.5f;
    float* fast = (float*)malloc(sizeof(float) * 12 * (size_t)k);
    if (!fast) return;
    oracle_fast_rows(rot12, off4, k, world, g, fast);
    for (int64_t p = 0; p < n; ++p) {
        const float* P = pos4 + 4 * p;
        const float cx = P[0] - half_l, cy = P[1] - half_l, cz = P[2] - half_l;
        for (int i = 0; i < k; ++i)
            cells[p * k + i] = cell_of(index_mode, rot12, off4, fast, i, cx, cy, cz, half_l, world,
                                       voxel, lg);
    }
    free(fast);
}

static uint64_t quantize_u64(float m, float scale) {
    const float v = m * scale;
    if (!(v >= 0.0f)) return 0;
    if (v >= 18446744073709551616.0f) return ~(uint64_t)0;
    return (uint64_t)v;
}
static uint32_t quantize_u32(float m) {
    const float v = m * 1000.0f; /* mass.glsl:54 */
    if (!(v >= 0.0f)) return 0;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}

/* Deposit into mass_out (k * g^3 cells, uint64 or uint32 per mode),
 * zeroed first.  Returns 0. */
ORACLE_API int oracle_deposit(const float* pos4, int64_t n, const float* rot12, const float* off4,
                              int k, int g, float world, int mass_mode, int scale_bits,
                              int index_mode, void* mass_out) {
    int lg = 0;
    while ((1 << lg) < g) ++lg;
    const float voxel = (float)((double)world / (double)g);
    const float half_l = world * 0.5f;
    const size_t g3 = (size_t)1 << (3 * lg);
    float* fast = (float*)malloc(sizeof(float) * 12 * (size_t)k);
    if (!fast) return 1;
    oracle_fast_rows(rot12, off4, k, world, g, fast);
    const float scale = ldexpf(1.0f, scale_bits);
    if (mass_mode == 0) memset(mass_out, 0, (size_t)k * g3 * 8);
    else memset(mass_out, 0, (size_t)k * g3 * 4);
    for (int64_t p = 0; p < n; ++p) {
        const float* P = pos4 + 4 * p;
        const float cx = P[0] - half_l, cy = P[1] - half_l, cz = P[2] - half_l;
        for (int i = 0; i < k; ++i) {
            const uint32_t c = cell_of(index_mode, rot12, off4, fast, i, cx, cy, cz, half_l,
                                       world, voxel, lg);
            if (mass_mode == 0)
                ((uint64_t*)mass_out)[(size_t)i * g3 + c] += quantize_u64(P[3], scale);
            else
                ((uint32_t*)mass_out)[(size_t)i * g3 + c] += quantize_u32(P[3]);
        }
    }
    free(fast);
    return 0;
}

/* update.glsl:53-89 from a grid-frame force grid (k * g^3 float4, the
 * reference's gradient texture layout).  When acc_out is non-null the
 * averaged force is written there instead of stepping. */
ORACLE_API int oracle_update(float* pos4, float* vel4, int64_t n, const float* force4,
                             const float* rot12, const float* off4, int k, int g, float world,
                             int index_mode, float dt, float damping, float* acc_out) {
    int lg = 0;
    while ((1 << lg) < g) ++lg;
    const float voxel = (float)((double)world / (double)g);
    const float half_l = world * 0.5f;
    const size_t g3 = (size_t)1 << (3 * lg);
    float* fast = (float*)malloc(sizeof(float) * 12 * (size_t)k);
    if (!fast) return 1;
    oracle_fast_rows(rot12, off4, k, world, g, fast);
    const float kf = (float)k;
    for (int64_t p = 0; p < n; ++p) {
        float* P = pos4 + 4 * p;
        const float cx = P[0] - half_l, cy = P[1] - half_l, cz = P[2] - half_l;
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (int i = 0; i < k; ++i) {
            const uint32_t c = cell_of(index_mode, rot12, off4, fast, i, cx, cy, cz, half_l,
                                       world, voxel, lg);
            const float* F = force4 + 4 * ((size_t)i * g3 + c);
            const float* R = rot12 + 12 * i;
            /* transpose(rot) * F = M F, update.glsl:77 */
            const float wx = (R[0] * F[0] + R[1] * F[1]) + R[2] * F[2];
            const float wy = (R[4] * F[0] + R[5] * F[1]) + R[6] * F[2];
            const float wz = (R[8] * F[0] + R[9] * F[1]) + R[10] * F[2];
            ax = ax + wx;
            ay = ay + wy;
            az = az + wz;
        }
        ax = ax / kf; /* update.glsl:81 */
        ay = ay / kf;
        az = az / kf;
        if (acc_out) {
            acc_out[4 * p + 0] = ax;
            acc_out[4 * p + 1] = ay;
            acc_out[4 * p + 2] = az;
            acc_out[4 * p + 3] = 0.0f;
            continue;
        }
        float* V = vel4 + 4 * p;
        float vx = V[0] - ax * dt, vy = V[1] - ay * dt, vz = V[2] - az * dt; /* :83 */
        vx = vx * damping;                                                   /* :84 */
        vy = vy * damping;
        vz = vz * damping;
        P[0] = glsl_mod(P[0] + vx * dt, world);                              /* :85-86 */
        P[1] = glsl_mod(P[1] + vy * dt, world);
        P[2] = glsl_mod(P[2] + vz * dt, world);
        V[0] = vx;
        V[1] = vy;
        V[2] = vz;
        V[3] = 0.0f;
    }
    free(fast);
    return 0;
}

/* Cell value as float, as the solver reads it (complex.glsl:23 for u32). */
ORACLE_API void oracle_mass_values(const void* mass, int64_t cells, int mass_mode, int scale_bits,
                                   float* out) {
    const float inv = ldexpf(1.0f, -scale_bits);
    for (int64_t c = 0; c < cells; ++c) {
        if (mass_mode == 0) out[c] = (float)((const uint64_t*)mass)[c] * inv;
        else out[c] = (float)((const uint32_t*)mass)[c] / 1000.0f;
    }
}
