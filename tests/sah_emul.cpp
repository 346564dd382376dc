// A host build of the device SAH builder's per-node code
// (phiray_b200/csrc/sah_core.cuh): the same steps phx_bvh_build_sah
// launches, run as loops over each level's nodes, so the CPU tests check
// the device code's arithmetic and its tree numbering against the oracle.
#include <cstring>
#include <vector>

#include "../phiray_b200/csrc/sah_core.cuh"

using namespace phx::sah;

extern "C" uint32_t emul_build_sah(const float* prims, uint32_t n, uint32_t leaf, float* nodes, uint32_t* order,
                                   uint32_t* depth) {
    *depth = 0;
    if (n == 0) return 0;
    const uint32_t cap = 2 * n - 1;
    std::vector<float> centres(3 * (size_t)n);
    for (uint32_t i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) centres[3 * (size_t)i + k] = 0.5f * (prims[8 * (size_t)i + k] + prims[8 * (size_t)i + 4 + k]);
        order[i] = i;
    }
    std::vector<TNode> tn(cap);
    std::vector<uint32_t> lists(cap), inner(cap), rank(cap), final_index(cap);
    std::vector<Box> boxes(cap);
    tn[0] = TNode{0, n, 0, NONE, NONE};
    lists[0] = 0;
    rank[0] = 0;
    final_index[0] = 0;
    uint32_t tcount = 1;
    auto add = [](uint32_t* p, uint32_t v) {
        const uint32_t old = *p;
        *p += v;
        return old;
    };
    std::vector<uint32_t> off{0}, len{1};
    for (uint32_t lv = 0; lv < MAX_DEPTH; lv++) {
        const uint32_t next = off[lv] + len[lv];
        uint32_t opened = 0;
        for (uint32_t k = 0; k < len[lv]; k++)
            process(lists[off[lv] + k], tn.data(), prims, centres.data(), order, leaf, &tcount,
                    lists.data() + next, &opened, add);
        if (opened == 0) break;
        off.push_back(next);
        len.push_back(opened);
    }
    const uint32_t levels = (uint32_t)len.size();
    for (uint32_t lv = levels; lv-- > 0;)
        for (uint32_t k = 0; k < len[lv]; k++) count_inner(lists[off[lv] + k], tn.data(), inner.data());
    for (uint32_t lv = 0; lv < levels; lv++)
        for (uint32_t k = 0; k < len[lv]; k++)
            place(lists[off[lv] + k], tn.data(), inner.data(), rank.data(), final_index.data());
    for (uint32_t lv = levels; lv-- > 0;)
        for (uint32_t k = 0; k < len[lv]; k++)
            emit(lists[off[lv] + k], tn.data(), final_index.data(), prims, order, boxes.data(), nodes);
    *depth = levels - 1;
    return tcount;
}
