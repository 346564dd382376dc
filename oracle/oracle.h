/*
 * ORACLE — test infrastructure only. A CPU restatement, in C++, of
 * gemphi/phiray's own CPU twins and WGSL for the Rendered-mode hot path.
 * The reference is Rust + WGSL and cannot be built or run here (no Rust
 * toolchain, no graphics stack), so this restatement is the checker the
 * CUDA kernels are compared against, and the CPU baseline bench.py times.
 * Nothing in the product links or calls it.
 *
 * Every function cites the reference file:line it follows. Pinned against
 * the reference's own test vectors (see tests/test_oracle_*.py).
 */
#ifndef PHIRAY_ORACLE_H
#define PHIRAY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_aabb {
    float lo[3];
    float pad_a;
    float hi[3];
    float pad_b;
} orc_aabb;

typedef struct orc_half {
    float p[3];
    uint32_t i;
} orc_half;

typedef struct orc_node {
    orc_half lo, hi;
} orc_node;

typedef struct orc_link {
    uint32_t left, right, first, last;
} orc_link;

typedef struct orc_pair {
    uint32_t bone;
    float weight;
    uint32_t next;
    float blend;
} orc_pair;

int orc_threads(void);
void orc_set_threads(int n);

/* src/bvh/node.rs:96-105 morton(p, group) (64-bit, group in the high word). */
uint64_t orc_morton(const float p[3], uint32_t group);
/* src/bvh/build.rs:70-72 Bvh::scene. */
void orc_scene(const orc_aabb* prims, uint32_t n, orc_aabb* out);
/* src/bvh/build.rs:75-85 Bvh::codes. */
void orc_codes(const orc_aabb* prims, uint32_t n, uint32_t* codes);
/* src/bvh/build.rs:87-92 Bvh::sort_codes: order by (code, index). */
void orc_sort_codes(const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted);
/* src/bvh/sort.rs:127-150: the reference's sequential model of its GPU
 * radix (8 LSD passes over the 64-bit key [index, code]). */
void orc_radix_model(const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted);
/* src/bvh/mod.rs:33-43 delta. */
int32_t orc_delta(const uint32_t* codes, uint32_t n, int64_t i, int64_t j);
/* src/bvh/build.rs:28-60 Link::of, for every internal node (n-1 links). */
void orc_links(const uint32_t* sorted, uint32_t n, orc_link* links);
/* src/bvh/build.rs:139-168 Bvh::assemble: nodes (2n-1), depth. */
void orc_assemble(uint32_t n, const orc_link* links, uint32_t leaf, orc_node* nodes, uint32_t* depth);
/* src/bvh/build.rs:180-194 Bvh::refit over `prims` through `order`. */
void orc_refit(orc_node* nodes, uint32_t nnodes, const uint32_t* order, const orc_aabb* prims);
/* src/bvh/build.rs:94-100 Bvh::build: nodes (2n-1), order (n), depth. */
void orc_build(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* nodes, uint32_t* order, uint32_t* depth);
/* src/bvh/build.rs:104-136 Bvh::build_compact; returns the node count
 * (nodes must hold 2n-1). */
uint32_t orc_build_compact(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* nodes, uint32_t* order,
                           uint32_t* depth);
/* src/bvh/sah.rs:84-189 Bvh::build_sah, the binned SAH tree phiray's tracer
 * walks: nodes (room for 2n-1), order (n), depth; returns the node count. */
uint32_t orc_build_sah(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* nodes, uint32_t* order,
                       uint32_t* depth);
/* src/bvh/shape.rs:8-37 Bvh::compact in place; returns the new count. */
uint32_t orc_compact(orc_node* nodes, uint32_t nnodes);
/* src/bvh/shape.rs:40-51 Bvh::reachable; returns the count written. */
uint32_t orc_reachable(const orc_node* nodes, uint32_t nnodes, uint32_t* out);

/* src/kernel/skin.rs:70-90 Skin::cpu. rest/out: vec4 x n; bones mat4 x k. */
void orc_skin(const float* rest, const uint32_t* offsets, const orc_pair* pairs, const float* bones, float min,
              uint32_t n, float* out);

/* src/kernel/denoise.wgsl:47-134 + view.wgsl:62-99, run as
 * Tracer::denoise_with (src/trace/read.rs:85-119) runs it: four passes,
 * steps 1, 2, 4, 8, in place on a px buffer of 34 w h + 1 words. */
void orc_denoise(uint32_t* px, uint32_t w, uint32_t h, const float strength[4], const float view[4], int keep);

/* The Rendered-mode tracer (shade.wgsl main and what it calls) over one
 * identity-instance scene: verts (x, y, z, 1) x V, faces (v0, v1, v2, mat)
 * x F, mats 32 words (trace::Mat) each, optional vertex normals, LBVH leaf
 * size. Frames [first, first + spp) of `cam` (a phx_camera, the reference's
 * Camera) accumulated into px (34 w h + 1 words, in/out), rows
 * [row0, row0 + rows) (rows 0 = all). *rays_out = rays traced. */
struct phx_camera;
void orc_trace(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, const float* normals,
               uint32_t leaf, const struct phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
               uint64_t* rays_out, uint32_t row0, uint32_t rows);
/* The same with the scene (tree, emitter table) built once. */
void* orc_scene_new(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, const float* normals,
                    uint32_t leaf);
void orc_scene_free(void* scene);
void orc_scene_trace(void* scene, const struct phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                     uint64_t* rays_out, uint32_t row0, uint32_t rows);
/* The same scene with the binned SAH tree (sah.rs) in place of the Morton one. */
void* orc_scene_new_sah(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats,
                        const float* normals, uint32_t leaf);
/* orc_scene_trace that also counts the walks' inner-node visits (walk[0]) and
 * triangle tests (walk[1]). */
void orc_scene_trace_walk(void* scene, const struct phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                          uint64_t* rays, uint32_t row0, uint32_t rows, uint64_t* walk);
/* Primary ray of frame `frame` per pixel: face id (0xFFFFFFFF none), t. */
// show.wgsl: emit's display tail (shown planes, packed pixels) over the sums in px.
void orc_show(const struct phx_camera* cam, uint32_t* px);
void orc_primary(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, uint32_t leaf,
                 const struct phx_camera* cam, uint32_t frame, uint32_t* ids, float* ts);
/* Closest / any hit of rays (o.xyz, tmax, d.xyz, 0): hits (t, face id, u, v). */
void orc_trace_rays(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, uint32_t leaf,
                    const float* rays, uint32_t n, float* hits, int any_hit);

/* tri.rs:51-114: the watertight test of one ray against one triangle;
 * returns 1 with out = (t, u, v) on a hit. */
int orc_tri_hit(const float* a, const float* b, const float* c, const float* o, const float* d, float* out);
/* phiray_math.h on the host: fn 0 exp2, 1 log2, 2 sin, 3 cos, 4 pow, 5 exp. */
void orc_math(int fn, const float* x, const float* y, float* out, uint32_t n);

#ifdef __cplusplus
}
#endif

#endif
