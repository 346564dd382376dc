// ORACLE — test infrastructure only (see oracle.h). CPU restatement of
// phiray's a-trous Denoise: src/kernel/denoise.wgsl:1-134 with
// denoise_param.wgsl, view.wgsl:62-99, driven as Tracer::denoise_with
// (src/trace/read.rs:85-119) drives it: steps 1, 2, 4, 8, round = pass.
#include <cstring>
#include <vector>

#include "oracle.h"
#include "wgsl.h"

using namespace wg;

namespace {

struct Den {
    uint32_t* px;
    uint32_t n, w, h, step, round, last, keep;
    float strength[4];
    float view[4];

    float f_at(uint32_t i) const { return wg::f_of(px[i]); }
    V3 v3_at(uint32_t base, uint32_t i) const {
        const uint32_t o = base + 3 * i;
        return v3(f_at(o), f_at(o + 1), f_at(o + 2));
    }
    void put3(uint32_t base, uint32_t i, V3 v) {
        const uint32_t o = base + 3 * i;
        px[o] = u_of(v.x);
        px[o + 1] = u_of(v.y);
        px[o + 2] = u_of(v.z);
    }
    // denoise.wgsl:23
    float inv_n(uint32_t i) const {
        const uint32_t c = px[31 * n + i];
        return 1.0f / (float)(c > 1 ? c : 1);
    }
    // denoise.wgsl:31-33
    V3 albedo_of(uint32_t i) const { return srgb(v3_at(7 * n, i) * inv_n(i)); }
    V3 normal_of(uint32_t i) const { return normalize(v3_at(10 * n, i) + v3(1e-9f)); }
    float depth_of(uint32_t i) const { return f_at(13 * n + i) * inv_n(i); }
    // denoise.wgsl:37-39
    V3 demodulated(uint32_t i) const { return v3_at(1 * n, i) * inv_n(i) / vmax(albedo_of(i), v3(0.05f)); }
    // denoise.wgsl:41-44
    V3 read_in(uint32_t i) const {
        if (round == 0) return demodulated(i);
        return v3_at(((round & 1) == 1 ? 14u : 17u) * n, i);
    }
    static float luma_of(V3 c) { return dot(c, v3(0.2126f, 0.7152f, 0.0722f)); }

    // denoise.wgsl:51-134 for pixel i, writing into `out` (a copy of px:
    // every plane a pass writes is one no other pixel of the pass reads).
    void pixel(uint32_t i, uint32_t* out) const {
        static const float KERNEL[3] = {0.375f, 0.25f, 0.0625f};
        const int x = (int)(i % w), y = (int)(i / w);
        V3 centre = read_in(i);
        if (round == 0) {
            float near_top = 0.0f;
            V3 near_sum = v3(0.0f);
            float near_n = 0.0f;
            for (int dy = -1; dy <= 1; dy++) {
                for (int dx = -1; dx <= 1; dx++) {
                    const int sx = x + dx, sy = y + dy;
                    if ((dx == 0 && dy == 0) || sx < 0 || sy < 0 || sx >= (int)w || sy >= (int)h) continue;
                    const V3 c = read_in((uint32_t)sy * w + (uint32_t)sx);
                    near_top = fmaxw(near_top, luma_of(c));
                    near_sum += c;
                    near_n += 1.0f;
                }
            }
            if (near_n > 0.0f && luma_of(centre) > 1.5f * near_top + 0.05f) centre = near_sum / near_n;
        }
        const V3 cn = normal_of(i);
        const V3 ca = albedo_of(i);
        const float cd = depth_of(i);
        const float lc = luma_of(centre);
        V3 sum = v3(0.0f);
        float weight = 0.0f;
        for (int dy = -2; dy <= 2; dy++) {
            for (int dx = -2; dx <= 2; dx++) {
                const int sx = x + dx * (int)step, sy = y + dy * (int)step;
                if (sx < 0 || sy < 0 || sx >= (int)w || sy >= (int)h) continue;
                const uint32_t j = (uint32_t)sy * w + (uint32_t)sx;
                if ((depth_of(j) < 0.0f) != (cd < 0.0f)) continue;
                const V3 tap = (j == i) ? centre : read_in(j);
                const float dn = fmaxw(0.0f, 1.0f - dot(cn, normal_of(j)));
                const float da = length(albedo_of(j) - ca);
                const float dd = std::fabs(depth_of(j) - cd) / fmaxw(std::fabs(cd), 1e-3f);
                const float dl = std::fabs(luma_of(tap) - lc) / (0.08f + lc);
                const float stop = pm_exp(-dn * strength[0] - da * strength[1] - dd * strength[2] -
                                          dl * dl * strength[3]);
                const float k = KERNEL[dx < 0 ? -dx : dx] * KERNEL[dy < 0 ? -dy : dy];
                sum += tap * k * stop;
                weight += k * stop;
            }
        }
        const V3 outv = weight > 0.0f ? sum / weight : centre;
        auto put = [&](uint32_t base, V3 v) {
            const uint32_t o = base + 3 * i;
            out[o] = u_of(v.x);
            out[o + 1] = u_of(v.y);
            out[o + 2] = u_of(v.z);
        };
        if (last == 0) {
            put(((round & 1) == 1 ? 17u : 14u) * n, outv);
            return;
        }
        const float k = inv_n(i);
        const float met = 1.0f - f_at(33 * n + i) * k;
        const V3 lin = (met > 0.5f * k) ? outv * vmax(albedo_of(i), v3(0.05f)) : v3(0.0f);
        if (keep == 0) put(1 * n, lin / k);
        const float cov = f_at(23 * n + i) * k;
        const V3 grid = v3_at(20 * n, i) * k;
        const V3 shown = view_transform_of(lin / fmaxw(met, k), view) * (1.0f - cov) + grid;
        put(4 * n, shown);
        out[i] = pack(shown, f_at(24 * n + i) * k);
    }
};

}  // namespace

extern "C" void orc_denoise(uint32_t* px, uint32_t w, uint32_t h, const float strength[4], const float view[4],
                            int keep) {
    const uint32_t n = w * h;
    if (n == 0) return;
    const uint32_t steps[4] = {1, 2, 4, 8};
    std::vector<uint32_t> out((size_t)34 * n + 1);
    for (uint32_t r = 0; r < 4; r++) {
        Den d;
        d.px = px;
        d.n = n;
        d.w = w;
        d.h = h;
        d.step = steps[r];
        d.round = r;
        d.last = steps[r] == 8 ? 1 : 0;
        d.keep = keep ? 1 : 0;
        std::memcpy(d.strength, strength, sizeof d.strength);
        std::memcpy(d.view, view, sizeof d.view);
        std::memcpy(out.data(), px, out.size() * 4);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < (int64_t)n; i++) d.pixel((uint32_t)i, out.data());
        std::memcpy(px, out.data(), out.size() * 4);
    }
}
