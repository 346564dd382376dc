// ORACLE — test infrastructure only (see oracle.h). WGSL's vector built-ins
// with one fixed evaluation order, so the restatement of a shader computes
// each expression the way the shader writes it: dot is ((x + y) + z),
// normalize divides by the length, mix is a (1 - t) + b t (the WGSL spec's
// formula), select(f, t, c) picks t when c holds.
#ifndef PHIRAY_ORACLE_WGSL_H
#define PHIRAY_ORACLE_WGSL_H

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../include/phiray_math.h"

namespace wg {

struct V3 {
    float x, y, z;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 v3(float s) { return V3{s, s, s}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3& operator+=(V3& a, V3 b) { return a = a + b; }
inline V3& operator*=(V3& a, V3 b) { return a = a * b; }
inline V3& operator*=(V3& a, float s) { return a = a * s; }

inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) {
    const float l = length(a);
    return {a.x / l, a.y / l, a.z / l};
}
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float fmaxw(float a, float b) { return std::fmax(a, b); }
inline float fminw(float a, float b) { return std::fmin(a, b); }
inline V3 vmax(V3 a, V3 b) { return {fmaxw(a.x, b.x), fmaxw(a.y, b.y), fmaxw(a.z, b.z)}; }
inline V3 vmin(V3 a, V3 b) { return {fminw(a.x, b.x), fminw(a.y, b.y), fminw(a.z, b.z)}; }
inline float clampf(float x, float lo, float hi) { return fminw(fmaxw(x, lo), hi); }
inline V3 vclamp(V3 a, float lo, float hi) { return {clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi)}; }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 vmix(V3 a, V3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
inline V3 vmix(V3 a, V3 b, V3 t) { return {mixf(a.x, b.x, t.x), mixf(a.y, b.y, t.y), mixf(a.z, b.z, t.z)}; }
inline float maxc(V3 a) { return fmaxw(a.x, fmaxw(a.y, a.z)); }
inline V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline float smoothstep(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline V3 reflect(V3 e1, V3 e2) { return e1 - e2 * (2.0f * dot(e2, e1)); }
// WGSL refract(e1, e2, e3): k = 1 - e3^2 (1 - dot(e2,e1)^2); 0 if k < 0,
// else e3 e1 - (e3 dot(e2,e1) + sqrt(k)) e2.
inline V3 refract(V3 e1, V3 e2, float e3) {
    const float d = dot(e2, e1);
    const float k = 1.0f - e3 * e3 * (1.0f - d * d);
    if (k < 0.0f) return v3(0.0f);
    return e1 * e3 - e2 * (e3 * d + std::sqrt(k));
}

inline float f_of(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t u_of(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// view.wgsl:88-93 srgb. 1/2.4 is written as the float nearest to it.
inline float srgb1(float c) {
    const float x = clampf(c, 0.0f, 1.0f);
    const float lo = x * 12.92f;
    const float hi = 1.055f * pm_pow(x, 0.416666657f) - 0.055f;
    return x <= 0.0031308f ? lo : hi;
}
inline V3 srgb(V3 c) { return {srgb1(c.x), srgb1(c.y), srgb1(c.z)}; }

// view.wgsl:62-85 view_transform_of, the Standard transform (kind 0).
inline V3 view_transform_of(V3 lin, const float view[4]) {
    const V3 c = vmax(lin, v3(0.0f)) * pm_exp2(view[1]);
    V3 d = srgb(c);
    float g = view[2];
    if (g <= 0.0f) g = 1.0f;
    const float e = 1.0f / g;
    const V3 cl = vclamp(d, 0.0f, 1.0f);
    return {pm_pow(cl.x, e), pm_pow(cl.y, e), pm_pow(cl.z, e)};
}

// view.wgsl:95-99 pack.
inline uint32_t pack(V3 c, float a) {
    const V3 q = vclamp(c, 0.0f, 1.0f) * 255.0f;
    const uint32_t r = (uint32_t)(q.x + 0.5f), g = (uint32_t)(q.y + 0.5f), b = (uint32_t)(q.z + 0.5f);
    const uint32_t qa = (uint32_t)(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f);
    return r | (g << 8) | (b << 16) | (qa << 24);
}

}  // namespace wg

#endif
