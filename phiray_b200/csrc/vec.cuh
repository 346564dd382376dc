// Device vector helpers with WGSL's built-ins in one fixed evaluation order
// (dot is ((x + y) + z), normalize divides by the length, mix is
// a (1 - t) + b t), so a kernel computes each expression as phiray's shader
// writes it. Kernels that include this are built with --fmad=false.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/phiray_math.h"

namespace phx {

struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 mk(float s) { return f3{s, s, s}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, f3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ f3& operator+=(f3& a, f3 b) { return a = a + b; }
__host__ __device__ __forceinline__ f3& operator*=(f3& a, f3 b) { return a = a * b; }
__host__ __device__ __forceinline__ f3& operator*=(f3& a, float s) { return a = a * s; }

__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ f3 normalize(f3 a) {
    const float l = length(a);
    return {a.x / l, a.y / l, a.z / l};
}
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ f3 vmax(f3 a, f3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__host__ __device__ __forceinline__ f3 vmin(f3 a, f3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__host__ __device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__host__ __device__ __forceinline__ f3 vclamp(f3 a, float lo, float hi) {
    return {clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi)};
}
__host__ __device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__host__ __device__ __forceinline__ f3 vmix(f3 a, f3 b, float t) {
    return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)};
}
__host__ __device__ __forceinline__ f3 vmix(f3 a, f3 b, f3 t) {
    return {mixf(a.x, b.x, t.x), mixf(a.y, b.y, t.y), mixf(a.z, b.z, t.z)};
}
__host__ __device__ __forceinline__ float maxc(f3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__host__ __device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
__host__ __device__ __forceinline__ f3 reflect(f3 e1, f3 e2) { return e1 - e2 * (2.0f * dot(e2, e1)); }
__host__ __device__ __forceinline__ f3 refract(f3 e1, f3 e2, float e3) {
    const float d = dot(e2, e1);
    const float k = 1.0f - e3 * e3 * (1.0f - d * d);
    if (k < 0.0f) return mk(0.0f);
    return e1 * e3 - e2 * (e3 * d + sqrtf(k));
}

// view.wgsl:88-93 srgb (1/2.4 as the float nearest to it).
__host__ __device__ __forceinline__ float srgb1(float c) {
    const float x = clampf(c, 0.0f, 1.0f);
    const float lo = x * 12.92f;
    const float hi = 1.055f * pm_pow(x, 0.416666657f) - 0.055f;
    return x <= 0.0031308f ? lo : hi;
}
__host__ __device__ __forceinline__ f3 srgb(f3 c) { return {srgb1(c.x), srgb1(c.y), srgb1(c.z)}; }

// view.wgsl:62-85 view_transform_of, Standard (view[0] == 0).
__host__ __device__ __forceinline__ f3 view_transform_std(f3 lin, float exposure, float gamma) {
    const f3 c = vmax(lin, mk(0.0f)) * pm_exp2(exposure);
    const f3 d = srgb(c);
    float g = gamma;
    if (g <= 0.0f) g = 1.0f;
    const float e = 1.0f / g;
    const f3 cl = vclamp(d, 0.0f, 1.0f);
    return {pm_pow(cl.x, e), pm_pow(cl.y, e), pm_pow(cl.z, e)};
}

// view.wgsl:95-99 pack.
__host__ __device__ __forceinline__ uint32_t pack_rgba(f3 c, float a) {
    const f3 q = vclamp(c, 0.0f, 1.0f) * 255.0f;
    const uint32_t r = (uint32_t)(q.x + 0.5f), g = (uint32_t)(q.y + 0.5f), b = (uint32_t)(q.z + 0.5f);
    const uint32_t qa = (uint32_t)(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f);
    return r | (g << 8) | (b << 16) | (qa << 24);
}

}  // namespace phx
