// ORACLE — test infrastructure only (see oracle.h). CPU restatement of
// phiray's Skin::cpu, src/kernel/skin.rs:70-90, in its own operation order.
#include "oracle.h"

extern "C" void orc_skin(const float* rest, const uint32_t* offsets, const orc_pair* pairs, const float* bones,
                         float min, uint32_t n, float* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float* r = rest + 4 * i;
        float acc[3] = {0.0f, 0.0f, 0.0f};
        float total = 0.0f;
        for (uint32_t q = offsets[i]; q < offsets[i + 1]; q++) {
            const orc_pair& p = pairs[q];
            const float* m = bones + 16 * (uint64_t)p.bone;
            const float* nx = bones + 16 * (uint64_t)p.next;
            auto at = [&](int j) { return m[j] + (nx[j] - m[j]) * p.blend; };
            for (int k = 0; k < 3; k++) {
                acc[k] += p.weight * (at(k) * r[0] + at(4 + k) * r[1] + at(8 + k) * r[2] + at(12 + k));
            }
            total += p.weight;
        }
        float* o = out + 4 * i;
        if (total > min) {
            o[0] = acc[0] / total;
            o[1] = acc[1] / total;
            o[2] = acc[2] / total;
        } else {
            o[0] = r[0];
            o[1] = r[1];
            o[2] = r[2];
        }
        o[3] = 1.0f;
    }
}
