// Linear blend skinning over CSR influences (phiray kernel::Skin,
// src/kernel/skin.rs:34-90) and the face boxes a refit reads
// (Pose::boxes, src/trace/pose.rs:45-51).
//
// One thread per vertex; the bone matrices are staged in shared memory once
// per block (64 B each), the CSR pairs read as one 16-byte load each. The
// arithmetic follows Skin::cpu's order, `at(k) r0 + at(4+k) r1 + at(8+k) r2 +
// at(12+k)` then `/ total`, built without contraction, so the output is the
// CPU twin's bit for bit.
#include "internal.cuh"

namespace phx {
namespace {

constexpr uint32_t SMEM_BONES = 512;  // 32 KB of matrices staged per block

template <bool STAGED>
__global__ void __launch_bounds__(256) k_skin(const float4* __restrict__ rest, const uint32_t* __restrict__ offsets,
                                              const uint4* __restrict__ pairs, const float4* __restrict__ bones,
                                              uint32_t nbones, float4* __restrict__ out, uint32_t n, float min,
                                              uint32_t* status) {
    __shared__ float4 s_bones[STAGED ? SMEM_BONES * 4 : 1];
    if (STAGED) {
        for (uint32_t k = threadIdx.x; k < nbones * 4; k += blockDim.x) s_bones[k] = __ldg(bones + k);
        __syncthreads();
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r = __ldg(rest + i);
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f, total = 0.0f;
    const uint32_t q0 = __ldg(offsets + i), q1 = __ldg(offsets + i + 1);
    bool bad = false;
    for (uint32_t q = q0; q < q1; q++) {
        const uint4 pr = __ldg(pairs + q);
        const uint32_t bone = pr.x, next = pr.z;
        const float w = __uint_as_float(pr.y), blend = __uint_as_float(pr.w);
        if (bone >= nbones || next >= nbones) {
            bad = true;
            continue;
        }
        float m[16], x[16];
        for (int c = 0; c < 4; c++) {
            const float4 a = STAGED ? s_bones[bone * 4 + c] : __ldg(bones + bone * 4 + c);
            const float4 b = STAGED ? s_bones[next * 4 + c] : __ldg(bones + next * 4 + c);
            m[4 * c + 0] = a.x;
            m[4 * c + 1] = a.y;
            m[4 * c + 2] = a.z;
            m[4 * c + 3] = a.w;
            x[4 * c + 0] = b.x;
            x[4 * c + 1] = b.y;
            x[4 * c + 2] = b.z;
            x[4 * c + 3] = b.w;
        }
        float at[16];
#pragma unroll
        for (int j = 0; j < 16; j++) at[j] = m[j] + (x[j] - m[j]) * blend;
        acc0 += w * (at[0] * r.x + at[4] * r.y + at[8] * r.z + at[12]);
        acc1 += w * (at[1] * r.x + at[5] * r.y + at[9] * r.z + at[13]);
        acc2 += w * (at[2] * r.x + at[6] * r.y + at[10] * r.z + at[14]);
        total += w;
    }
    if (bad) atomicOr(status, STATUS_BAD_INDEX);
    out[i] = total > min ? make_float4(acc0 / total, acc1 / total, acc2 / total, 1.0f) : make_float4(r.x, r.y, r.z, 1.0f);
}

// Aabb::of_tri (src/bvh/node.rs:79-81): a.min(b).min(c), a.max(b).max(c).
__global__ void __launch_bounds__(256) k_face_boxes(const float4* __restrict__ verts, const uint4* __restrict__ faces,
                                                    uint32_t nfaces, float4* __restrict__ boxes) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfaces) return;
    const uint4 v = __ldg(faces + f);
    const float4 a = __ldg(verts + v.x), b = __ldg(verts + v.y), c = __ldg(verts + v.z);
    boxes[2 * (size_t)f] = make_float4(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y),
                                       fminf(fminf(a.z, b.z), c.z), 0.0f);
    boxes[2 * (size_t)f + 1] = make_float4(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y),
                                           fmaxf(fmaxf(a.z, b.z), c.z), 0.0f);
}

int32_t launch_skin(cudaStream_t s, const float* rest, const uint32_t* offsets, const phx_pair* pairs,
                    const float* bones, uint32_t nbones, float* out, uint32_t n, float min, uint32_t* status) {
    if (n == 0) return PHX_OK;
    const uint32_t grid = (n + 255) / 256;
    if (nbones <= SMEM_BONES)
        k_skin<true><<<grid, 256, 0, s>>>((const float4*)rest, offsets, (const uint4*)pairs, (const float4*)bones,
                                          nbones, (float4*)out, n, min, status);
    else
        k_skin<false><<<grid, 256, 0, s>>>((const float4*)rest, offsets, (const uint4*)pairs, (const float4*)bones,
                                           nbones, (float4*)out, n, min, status);
    return cuda_check(cudaGetLastError(), "skin");
}

}  // namespace

int32_t launch_skin_step(cudaStream_t s, const void* params, void* const* bufs, const uint64_t* sizes, uint32_t items,
                         uint32_t* status) {
    phx_skin_param p;
    memcpy(&p, params, sizeof p);
    const uint32_t n = items < p.n ? items : p.n;
    const uint64_t nb = sizes[3] / 64;
    return launch_skin(s, (const float*)bufs[0], (const uint32_t*)bufs[1], (const phx_pair*)bufs[2],
                       (const float*)bufs[3], (uint32_t)(nb > 0xFFFFFFFFull ? 0xFFFFFFFFu : nb), (float*)bufs[4], n,
                       p.min, status);
}

int32_t launch_face_boxes(cudaStream_t s, const float* verts, const uint32_t* faces, uint32_t nfaces, phx_aabb* boxes) {
    if (nfaces == 0) return PHX_OK;
    k_face_boxes<<<(nfaces + 255) / 256, 256, 0, s>>>((const float4*)verts, (const uint4*)faces, nfaces, (float4*)boxes);
    return cuda_check(cudaGetLastError(), "face boxes");
}

}  // namespace phx

using namespace phx;

extern "C" {

int32_t phx_skin(phx_ctx ctx, const float* rest, const uint32_t* offsets, const phx_pair* pairs, const float* bones,
                 uint32_t nbones, float* out, uint32_t n, float min) {
    if (!ctx || (n && (!rest || !offsets || !out))) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(&ctx->c));
    return launch_skin(ctx->c.stream, rest, offsets, pairs, bones, nbones, out, n, min, ctx->c.status);
}

int32_t phx_face_boxes(phx_ctx ctx, const float* verts, const uint32_t* faces, uint32_t nfaces, phx_aabb* boxes) {
    if (!ctx || (nfaces && (!verts || !faces || !boxes))) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(&ctx->c));
    return launch_face_boxes(ctx->c.stream, verts, faces, nfaces, boxes);
}

}  // extern "C"
