/*
 * phiray_cuda.h — the C ABI of phiray-b200: phiray's Rendered-mode hot path
 * (LBVH build and refit, the 32-slot-stack path tracer, Skin, Denoise) as
 * CUDA kernels for sm_100a behind plain C entry points.
 *
 * Every entry point replaces a piece of phiray's Rust API (gemphi/phiray);
 * the citation beside each names the reference item it stands in for. A Rust
 * FFI crate binds these one for one (`extern "C"` blocks, no bindgen), and
 * wraps them in the same `Gpu`, `GpuArray`, `Pass`, `GpuBvh`, `Skin` and
 * `Tracer` types, so callers such as phiber's `RaySkin` and
 * `view3d/rendered.rs` keep their code.
 *
 * Conventions
 *   - Every call returns int32 status: PHX_OK (0), a positive informational
 *     code (PHX_REBUILD), or a negative PHX_ERR_*. The text of the last
 *     error on the calling thread is available from phx_last_error.
 *   - A context is one device and one CUDA stream; all work is stream-
 *     ordered on it. A context is used by one host thread at a time
 *     (phiray: `Gpu` is shared, `Tracer` is `&mut self`).
 *   - Every host wait is bounded by a timeout in milliseconds and fails with
 *     PHX_ERR_TIMEOUT instead of blocking forever (phiray `Gpu::wait_for`,
 *     src/gpu/mod.rs:292-303). timeout_ms 0 means the default patience
 *     (PHX_DEFAULT_WAIT_MS).
 *   - Device pointers are passed as `void*` / typed pointers to device
 *     memory; host pointers are documented as such.
 *   - There is no CPU fallback: without a CUDA device every call that needs
 *     one returns PHX_ERR_DEVICE.
 */
#ifndef PHIRAY_CUDA_H
#define PHIRAY_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (phiray: Option/bool "declined", empty readback) ---- */
#define PHX_OK 0
#define PHX_REBUILD 1          /* GpuBvh::update returned false: rebuild instead */
#define PHX_ERR_INVALID (-1)   /* bad argument (phiray panics on binding count)  */
#define PHX_ERR_OOM (-2)
#define PHX_ERR_TIMEOUT (-3)   /* phiray: empty readback, "device did not drain" */
#define PHX_ERR_CANCELLED (-4) /* phiray: sample_in's `go` said no               */
#define PHX_ERR_DEVICE (-5)    /* CUDA error, or no device                        */
#define PHX_ERR_KERNEL (-6)    /* a kernel reported a status word (bounded wait)  */

#define PHX_DEFAULT_WAIT_MS 5000u /* phiray WAIT_LIMIT, src/gpu/mod.rs:36 */

/* ---- shared layouts (byte-identical to the reference's Pod types) ---- */

/* bvh::Aabb, src/bvh/node.rs:60-66: 32 bytes, padded for WGSL. */
typedef struct phx_aabb {
    float lo[3];
    float pad_a;
    float hi[3];
    float pad_b;
} phx_aabb;

/* bvh::Half, src/bvh/node.rs:12-16: a bound corner + index with leaf bit 31. */
typedef struct phx_half {
    float p[3];
    uint32_t i;
} phx_half;

/* bvh::Node, src/bvh/node.rs:30-34. Inner: children lo.i, hi.i.
 * Leaf: sorted slots [lo.i & ~LEAF, hi.i). */
typedef struct phx_node {
    phx_half lo;
    phx_half hi;
} phx_node;

#define PHX_LEAF 0x80000000u /* bvh::LEAF, src/bvh/node.rs:7 */
#define PHX_STACK 32u        /* bvh::STACK, src/bvh/node.rs:6 */

/* bvh::Link, src/bvh/build.rs:8-14: Karras result for one internal node. */
typedef struct phx_link {
    uint32_t left, right, first, last;
} phx_link;

/* kernel::Pair, src/kernel/skin.rs:13-22. */
typedef struct phx_pair {
    uint32_t bone;
    float weight;
    uint32_t next;
    float blend;
} phx_pair;

/* ---- context (phiray Gpu, src/gpu/mod.rs:84-99) ---- */
typedef struct phx_ctx_s* phx_ctx;

/* Gpu::new: open device `ordinal`, create its stream. */
int32_t phx_ctx_create(int32_t ordinal, phx_ctx* out);
int32_t phx_ctx_destroy(phx_ctx ctx);
/* Gpu::wait_for (src/gpu/mod.rs:292-303): drain the stream, polling with a
 * deadline; PHX_ERR_TIMEOUT when it does not drain in time. */
int32_t phx_ctx_wait(phx_ctx ctx, uint32_t timeout_ms);
/* The cudaStream_t work is enqueued on (as void*). */
void* phx_ctx_stream(phx_ctx ctx);
/* Enqueue on a caller's stream (e.g. one shared with another library);
 * NULL returns to the context's own stream. */
int32_t phx_ctx_set_stream(phx_ctx ctx, void* stream);
/* The library's bounded device waits made to run out, for tests of the
 * failure path (no reference counterpart: phiray's WGSL never waits on
 * another invocation). which 0: the mbarrier wait of the tensor-core engine;
 * 1: the radix sort's look-back wait. The wait polls a flag nothing sets
 * (satisfied = 0) at most `limit` times, sets the context's status word and
 * returns; the call then reports PHX_ERR_KERNEL ("spin limit") and the
 * context stays usable. satisfied = 1 sets the flag first: PHX_OK. Waits. */
int32_t phx_selftest_wait(phx_ctx ctx, int32_t which, uint32_t limit, int32_t satisfied);
/* Text of the calling thread's last error; returns its length. */
int32_t phx_last_error(char* buf, size_t len);
/* Library version string, for loaders. */
const char* phx_version(void);
/* Number of CUDA devices (0 when none), no context needed. */
int32_t phx_device_count(void);

/* ---- buffers (phiray GpuArray<T>, src/gpu/array.rs:20-187) ---- */
typedef struct phx_buf_s* phx_buf;

/* GpuArray::new / zeroed: `bytes` of device memory, zeroed. */
int32_t phx_buf_alloc(phx_ctx ctx, uint64_t bytes, phx_buf* out);
/* Borrow caller-owned device memory as a buffer (not freed by phx_buf_free). */
int32_t phx_buf_wrap(phx_ctx ctx, void* device_ptr, uint64_t bytes, phx_buf* out);
int32_t phx_buf_free(phx_buf buf);
/* GpuArray::write_at (array.rs:99-107): host -> device, stream-ordered;
 * returns when `src` may be reused. */
int32_t phx_buf_write(phx_buf buf, uint64_t offset, const void* src, uint64_t bytes);
/* GpuArray::write (array.rs:47-56): replace the contents with `bytes` from
 * the host, reallocating when they do not fit; *reallocated = 1 then, which
 * (as in phiray) means passes bound to the old buffer must be re-added. */
int32_t phx_buf_assign(phx_buf buf, const void* src, uint64_t bytes, int32_t* reallocated);
/* GpuArray::read_range (array.rs:148-187): device -> host, bounded wait. */
int32_t phx_buf_read(phx_buf buf, uint64_t offset, void* dst, uint64_t bytes, uint32_t timeout_ms);
uint64_t phx_buf_size(phx_buf buf);
void* phx_buf_ptr(phx_buf buf);

/* ---- kernels and recorded passes (phiray Kernel + Pass) ---- */

/* Kernel ids stand in for Kernel::NAME/WGSL/key (src/kernel/mod.rs:51-105).
 * Each kernel's params blob starts with {n, groups_x} as phiray's Param does;
 * phx_pass_add fills those two words (Pass::add_over, src/gpu/pass.rs:70-101). */
enum phx_kernel_id {
    PHX_KERNEL_SKIN = 1,    /* kernel::Skin, src/kernel/skin.rs:34-66; params phx_skin_param; bufs rest, offsets, pairs, bones, out */
    PHX_KERNEL_DENOISE = 2, /* kernel::Denoise, src/kernel/denoise.rs:53-64; params phx_denoise_param; bufs px */
    PHX_KERNEL_MORTON = 3,  /* bvh::Morton, src/bvh/kernel.rs:21-51; params phx_morton_param; bufs prims, codes */
    PHX_KERNEL_KARRAS = 4,  /* bvh::Karras, src/bvh/kernel.rs:65-117; params phx_karras_param; bufs codes, links */
    PHX_KERNEL_REFIT = 5    /* bvh::Refit (one Jacobi step), src/bvh/kernel.rs:130-170; params phx_refit_param; bufs prims, order, src, dst */
};

/* kernel::SkinParam, src/kernel/skin.rs:24-32. */
typedef struct phx_skin_param {
    uint32_t n, groups_x;
    float min;
    uint32_t pad;
} phx_skin_param;

/* kernel::DenoiseParam, src/kernel/denoise.rs:24-51. */
typedef struct phx_denoise_param {
    uint32_t n, groups_x, w, h;
    uint32_t step, round, last, keep;
    float strength[4];
    float view[4];
} phx_denoise_param;

/* bvh::MortonParam, src/bvh/kernel.rs:9-18. */
typedef struct phx_morton_param {
    uint32_t n, groups_x, pad0[2];
    float lo[3];
    float pad1;
    float inv[3];
    float pad2;
} phx_morton_param;

/* bvh::KarrasParam, src/bvh/kernel.rs:55-62. */
typedef struct phx_karras_param {
    uint32_t n, groups_x, leaves, pad;
} phx_karras_param;

/* bvh::RefitParam, src/bvh/kernel.rs:121-126. */
typedef struct phx_refit_param {
    uint32_t n, groups_x, pad[2];
} phx_refit_param;

typedef struct phx_pass_s* phx_pass;

int32_t phx_pass_create(phx_ctx ctx, phx_pass* out);
int32_t phx_pass_destroy(phx_pass pass);
/* Pass::add_over (pass.rs:70-101): record kernel `id` over `items`
 * invocations of a job of `n`; `params` (params_len bytes) is copied, its
 * first two words set to {n, groups_x}. The buffer count must match the
 * kernel's (phiray asserts; this returns PHX_ERR_INVALID). *step = index. */
int32_t phx_pass_add(phx_pass pass, int32_t kernel_id, uint32_t n, uint32_t items, const void* params,
                     uint32_t params_len, const phx_buf* bufs, uint32_t nbufs, uint32_t* step);
/* Pass::set (pass.rs:104-106): overwrite `len` bytes of a step's params at
 * `offset`, stream-ordered before the next run. */
int32_t phx_pass_set(phx_pass pass, uint32_t step, uint32_t offset, const void* data, uint32_t len);
/* Pass::run (pass.rs:109-113): replay every step, as one CUDA graph launch. */
int32_t phx_pass_run(phx_pass pass);
/* Pass::run_step (pass.rs:126-137). */
int32_t phx_pass_run_step(phx_pass pass, uint32_t step);
/* Pass::clear (pass.rs:139). */
int32_t phx_pass_clear(phx_pass pass);
/* Pass::len. */
uint32_t phx_pass_len(phx_pass pass);
/* Pass::compiled: distinct kernels this pass uses. */
uint32_t phx_pass_compiled(phx_pass pass);

/* ---- GpuBvh (src/bvh/gpu.rs:11-104) ---- */
typedef struct phx_bvh_s* phx_bvh;

/* Bvh::build_sah (src/bvh/sah.rs:84-189) on the device: the binned SAH tree
 * phiray's tracer walks (forest.rs:49, 216), node for node — 16 centroid
 * bins per axis, the cheapest of the 45 planes, a leaf where splitting
 * costs more than testing what the node holds or at depth 31, the
 * reference's in-place partition of each node's slots and its node
 * numbering, bounds refit bottom up. All pointers are DEVICE memory:
 * prims (n phx_aabb), nodes (room for 2n - 1), order (n). Writes the node
 * count and depth; stream-ordered, waits once or twice per tree level.
 * Nodes under 64 slots are a thread's, 64-2,047 a block's, larger ones are
 * cut over blocks of 2,048 slots (1.3 M prims: ~9 ms). */
int32_t phx_bvh_build_sah(phx_ctx ctx, const phx_aabb* prims, uint32_t n, uint32_t leaf, phx_node* nodes,
                          uint32_t* order, uint32_t* node_count, uint32_t* depth);

/* GpuBvh::build (gpu.rs:23-74) from HOST prims: upload, then every stage on
 * the device — bounds, Morton codes, stable radix sort, Karras links, leaf
 * packing and depth, atomic bottom-up refit. No readback. n may be 0. */
int32_t phx_bvh_build(phx_ctx ctx, const phx_aabb* host_prims, uint32_t n, uint32_t leaf, phx_bvh* out);
/* The same from prims already in device memory (copied into the BVH). */
int32_t phx_bvh_build_device(phx_ctx ctx, const phx_aabb* device_prims, uint32_t n, uint32_t leaf, phx_bvh* out);
/* Rebuild an existing BVH in place over new prims (reuses its memory when
 * the count fits). */
int32_t phx_bvh_rebuild_device(phx_bvh bvh, const phx_aabb* device_prims, uint32_t n);
/* GpuBvh::refit (gpu.rs:88-90): bounds again from the BVH's prims. */
int32_t phx_bvh_refit(phx_bvh bvh);
/* GpuBvh::update (gpu.rs:93-99): new HOST prims of the same count, then
 * refit; PHX_REBUILD (no work done) when the count differs. */
int32_t phx_bvh_update(phx_bvh bvh, const phx_aabb* host_prims, uint32_t n);
/* The same with DEVICE prims. */
int32_t phx_bvh_update_device(phx_bvh bvh, const phx_aabb* device_prims, uint32_t n);
/* GpuBvh::download (gpu.rs:102-104): nodes (2n-1, host), order (n, host)
 * and depth. Either array may be NULL. Bounded wait. */
int32_t phx_bvh_download(phx_bvh bvh, phx_node* nodes, uint32_t* order, uint32_t* depth, uint32_t timeout_ms);
/* Counts: prims, node slots (2n-1), leaf size, depth (waits for the build). */
int32_t phx_bvh_info(phx_bvh bvh, uint32_t* n, uint32_t* nodes, uint32_t* leaf, uint32_t* depth);
/* Device pointers of the BVH's arrays (GpuBvh's pub fields prims, order,
 * nodes), plus the sorted Morton codes; any may be NULL. */
int32_t phx_bvh_device(phx_bvh bvh, phx_aabb** prims, uint32_t** order, phx_node** nodes, uint32_t** codes);
int32_t phx_bvh_destroy(phx_bvh bvh);

/* Stage-by-stage entry points over device arrays (the reference's GPU build
 * pieces, for tests and for callers that hold their own arrays). */
/* bvh::Morton (kernel.rs:21-51) with Bvh::scene (build.rs:70-72) done on the
 * device: codes[i] for prims[i]; scene box written to scene_out (device,
 * may be NULL). */
int32_t phx_morton(phx_ctx ctx, const phx_aabb* prims, uint32_t n, uint32_t* codes, phx_aabb* scene_out);
/* Bvh::sort_codes (build.rs:87-92) as a stable LSD radix sort: order[] and
 * sorted[] (device) equal to sorting (code, index). */
int32_t phx_sort_codes(phx_ctx ctx, const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted);
/* phx_sort_codes without allocating: no counterpart in the reference. For
 * callers that cannot allocate device memory at call time — a host that
 * hands the renderer a fixed, pre-reserved budget and owns every other byte
 * of the device, or a frame loop that must not stall on cudaMalloc/cudaFree
 * (both can wait for the whole device). The sort's working memory is one
 * array compiled into the library (~9.4 MB, held on every GPU that loads it
 * until the process exits), so n is at most PHX_SORT_STATIC_MAX (larger n:
 * PHX_ERR_INVALID, nothing launched). The first call on a device looks up
 * that array's device address and keeps it for the life of the process: do
 * not reset the device (cudaDeviceReset) while the library is loaded.
 * Stream-ordered and does not
 * wait: synchronise before reading order/sorted. A failure inside the sort's
 * kernels (a look-back wait that gave up) is reported by the next call that
 * reads the context's status, such as phx_ctx_wait. All calls share the
 * array, so calls whose work overlaps on the GPU (other streams, other host
 * threads) race. */
#define PHX_SORT_STATIC_MAX (1u << 20)
int32_t phx_sort_codes_static(phx_ctx ctx, const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted);
/* bvh::Karras (kernel.rs:65-117): links[i] for i < n-1 from sorted codes. */
int32_t phx_karras(phx_ctx ctx, const uint32_t* sorted, uint32_t n, phx_link* links);

/* ---- Skin (src/kernel/skin.rs) ---- */
/* kernel::Skin over device arrays: rest/out vec4 x n, offsets n+1, pairs,
 * bones (column-major mat4 x nbones). Pairs naming a bone >= nbones are an
 * error (PHX_ERR_KERNEL, from a status word the kernel sets). */
int32_t phx_skin(phx_ctx ctx, const float* rest, const uint32_t* offsets, const phx_pair* pairs, const float* bones,
                 uint32_t nbones, float* out, uint32_t n, float min);
/* Face boxes for a refit: box f = Aabb::of_tri of vertices faces[f].xyz
 * (phiray Pose::boxes, src/trace/pose.rs:45-51), from skinned positions. */
int32_t phx_face_boxes(phx_ctx ctx, const float* verts, const uint32_t* faces, uint32_t nfaces, phx_aabb* boxes);

/* ---- Denoise (src/kernel/denoise.rs, denoise.wgsl; Tracer::denoise_with,
 * src/trace/read.rs:85-119) ---- */
/* The four a-trous passes (steps 1, 2, 4, 8) over a px image of w*h pixels
 * (34 w h + 1 words, phiray's Tracer::PX_LEN layout, device). `strength`
 * and `view` as DenoiseParam; keep = Tracer::denoise_shown. Only the
 * Standard view transform (view[0] == 0) is supported. */
int32_t phx_denoise(phx_ctx ctx, uint32_t* px, uint32_t w, uint32_t h, const float strength[4], const float view[4],
                    int32_t keep);


/* ---- Tracer (src/trace/mod.rs, build.rs, sample.rs, read.rs) ---- */

/* camera.wgsl `Light` (src/trace/light.rs:15-43): 80 bytes. kind 0 sun,
 * 1 point, 2 spot, 3 area. */
typedef struct phx_light {
    float pos[3];
    uint32_t kind;
    float color[3];
    float size;
    float dir[3];
    float cone;
    float right[3];
    float size_y;
    uint32_t shape;
    float blend;
    float spot_scale[2];
} phx_light;

#define PHX_MAX_LIGHT 64

/* trace::Camera (src/trace/camera.rs:12-230, camera.wgsl:3-54), byte for
 * byte (5,776 bytes), so a Rust caller passes its `Camera` as is. The
 * Rendered path reads the view, lights, env, view transform, bounces,
 * limit and frame words; settings this library does not implement are
 * refused with PHX_ERR_INVALID (see phx_tracer_sample). */
typedef struct phx_camera {
    uint32_t n, groups_x, w, h;
    float right[3];
    uint32_t persp;
    float up[3];
    float scale;
    float back[3];
    float units;
    float pivot[3];
    float aspect;
    float sun[3];
    float dist;
    float sky[4];
    float pan[2];
    float ao, eps;
    uint32_t frame;
    float grid;
    uint32_t count, glow;
    float grid_color[4];
    float env[4];
    uint32_t split[4];
    float view[4];
    uint32_t envmap;
    float env_rot;
    uint32_t bounces, env_cdf;
    float aperture, focus;
    uint32_t blades;
    float blade_spin;
    float aperture_ratio;
    uint32_t env_hidden;
    float see_through;
    uint32_t grid_hide;
    uint32_t tile[4], film[4], preview[4], slice[4], insts[4], vis[4];
    float taa[4], fx[4], outline[4];
    uint32_t shade[4];
    float single[4], cavity[4];
    uint32_t ssao[4];
    float shadow[4], shadow_fade[4];
    uint32_t matcap[4];
    float dof[4], outline_fx[4], outline_pick[4], outline_active[4], outline_move[4];
    float adapt[4], limit[4];
    uint32_t depth[4];
    float integrator[4];
    phx_light lights[PHX_MAX_LIGHT];
} phx_camera;

/* A scene as indexed HOST arrays (what trace::Scene packs, scene.rs:41-64):
 * verts (nverts x 4 f32, xyz + 1), optional vertex normals (nverts x 4 f32,
 * zero = flat face; may be NULL), faces (nfaces x 4 u32: v0, v1, v2,
 * material), mats (nmats x 16 f32: color rgba, rough, metal, trans, ior,
 * emit rgb, then zeros — trace::Mat's Rendered-path inputs). */
typedef struct phx_scene {
    const float* verts;
    const float* normals;
    const uint32_t* faces;
    const float* mats;
    uint32_t nverts, nfaces, nmats;
    uint32_t leaf; /* LBVH leaf size (the tracer's 4, forest.rs:20) */
} phx_scene;

/* trace::Mesh (src/trace/mesh.rs:12-22): faces [face_lo, face_hi) of the
 * scene's face array, kept in the mesh's own space under a tree of its own. */
typedef struct phx_mesh {
    uint32_t face_lo, face_hi;
} phx_mesh;

/* trace::Instance (src/trace/instance.rs:20-37): one placement of a mesh.
 * world is object -> world in Blender's layout, m[col][row] at
 * world[4 * col + row] (translation in world[12..14]). casts_shadow 0: shadow
 * rays pass it (Cycles' Ray Visibility > Shadow). 32-byte aligned record. */
typedef struct phx_instance {
    float world[16];
    uint32_t mesh;
    uint32_t casts_shadow;
    uint32_t pad[6];
} phx_instance;

typedef struct phx_tracer_s* phx_tracer;

/* PX_LEN (src/trace/read.rs:56): words per pixel of the image buffer. */
#define PHX_PX_LEN 34u

/* Tracer::new (src/trace/build.rs:11-24): upload the scene, build its LBVH
 * on the device (the reference walks CPU-built SAH trees; here the GPU LBVH
 * is the tracer's tree), gather triangles into leaf order, build the
 * emitter table. */
int32_t phx_tracer_create(phx_ctx ctx, const phx_scene* scene, phx_tracer* out);
/* Tracer::new over meshes placed by instances (src/trace/forest.rs:44-61,
 * 126-158; instance.rs): each mesh's faces [face_lo, face_hi) get an LBVH of
 * their own in the mesh's space (the vertices stay there), the instances'
 * world boxes a top tree (one instance a leaf); the walk takes each ray
 * through the top tree and into each instance's mesh by its inverse
 * (bvh.wgsl:115-232), a hit remembers its instance, shading places the face
 * in the world by it (layout.wgsl tri_of, world_ng for mirroring matrices),
 * shadow rays pass instances that cast none, and the emitter table holds an
 * entry per (emissive face, instance) (lamp.rs table_of). Meshes must name
 * ascending, disjoint ranges; faces in no mesh are never hit. Vertex w is
 * taken as 1. */
int32_t phx_tracer_create_instanced(phx_ctx ctx, const phx_scene* scene, const phx_mesh* meshes, uint32_t nmeshes,
                                    const phx_instance* insts, uint32_t ninsts, phx_tracer* out);
/* Tracer::reinstance (src/trace/pose.rs:105-120): the same instances placed
 * by new matrices (and shadow flags); the top tree is rebuilt on the device,
 * the emitter table again, the image starts over. PHX_ERR_INVALID when the
 * count or an instance's mesh differs (build the tracer again) or the tracer
 * has no instances. Stream-ordered. */
int32_t phx_tracer_reinstance(phx_tracer tr, const phx_instance* insts, uint32_t ninsts);
int32_t phx_tracer_destroy(phx_tracer tr);
/* Which kernel traces a frame. All compute the same image bit for bit:
 * PHX_KERNEL_MEGAKERNEL (the default) is shade.wgsl's main as one thread per
 * pixel with the walk called from every site that traces;
 * PHX_KERNEL_STATE_MACHINE is a persistent kernel whose lanes take pixels from a
 * counter and run the bounce loop as a state machine around one walk, so
 * lanes at different points of their paths still traverse together. Its
 * _6 and _8 forms cap registers for 6 or 8 resident 128-thread blocks per
 * SM (more warps, path state spilled to local memory); phx_tracer_autotune
 * times them on the scene and keeps the fastest. */
#define PHX_KERNEL_MEGAKERNEL 0u
#define PHX_KERNEL_STATE_MACHINE 1u
#define PHX_KERNEL_STATE_MACHINE_6 2u
#define PHX_KERNEL_STATE_MACHINE_8 3u
/* The megakernel with a register budget for 3 or 2 resident blocks (more
 * registers a thread, fewer spills, fewer warps). */
#define PHX_KERNEL_MEGAKERNEL_3 4u
#define PHX_KERNEL_MEGAKERNEL_2 5u
/* The megakernel (4 or 2 resident blocks) with each warp's lanes waiting for
 * each other after every sample, so samples start together. */
#define PHX_KERNEL_MEGAKERNEL_SYNC 6u
#define PHX_KERNEL_MEGAKERNEL_2_SYNC 7u
/* The megakernel with a register budget for 5, 6 or 8 resident blocks (more
 * warps to hide the walk's load latency, more spills), and the 6- and
 * 8-block forms with the per-sample warp wait. */
#define PHX_KERNEL_MEGAKERNEL_5 8u
#define PHX_KERNEL_MEGAKERNEL_6 9u
#define PHX_KERNEL_MEGAKERNEL_6_SYNC 10u
#define PHX_KERNEL_MEGAKERNEL_8 11u
#define PHX_KERNEL_MEGAKERNEL_8_SYNC 12u
/* The same with the per-sample warp wait at 10, 12 and 16 resident blocks
 * (48, 40 and 32 registers a thread). */
#define PHX_KERNEL_MEGAKERNEL_10_SYNC 13u
#define PHX_KERNEL_MEGAKERNEL_12_SYNC 14u
#define PHX_KERNEL_MEGAKERNEL_16_SYNC 15u
/* The wavefront render: path state in device memory, rays queued by type
 * (primary, extension, shadow) with ballot compaction, each queue walked by a
 * kernel of its own (closest or any hit) between passes of the shading
 * logic; the host polls the queues every fourth pass. Not inside a graph
 * capture nor with adaptive sampling (the megakernel runs those frames). */
#define PHX_KERNEL_WAVEFRONT 16u
/* The megakernel whose walk keeps the top of its 32-entry stack in
 * registers (older entries spill to local memory, a pop refilling the
 * registers ahead of use): 8 register entries at 4 resident blocks (128
 * registers a thread), the top entry at 8 and at 16 resident blocks with the
 * per-sample warp wait. */
#define PHX_KERNEL_MEGAKERNEL_REG 17u
#define PHX_KERNEL_MEGAKERNEL_8_SYNC_REG 18u
#define PHX_KERNEL_MEGAKERNEL_16_SYNC_REG 19u
/* Number of render kernel ids (the length of phx_tracer_autotune's ms). */
#define PHX_KERNEL_COUNT 20u
int32_t phx_tracer_set_kernel(phx_tracer tr, uint32_t kernel);
/* The autotuner: times every render kernel (and register budget) above on
 * `spp` samples of this scene and camera, keeps the fastest for the tracer
 * and returns its id; ms (PHX_KERNEL_COUNT floats, may be NULL) gets each one's time. The
 * image is overwritten (the next sample starts over). Waits. */
int32_t phx_tracer_autotune(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t spp,
                            uint32_t* chosen, float* ms);
/* Where thread-per-ray walks (phx_trace_rays under PHX_WALK_THREAD) keep
 * their 32-entry stack: PHX_STACK_LOCAL (per-thread local memory, the
 * default), PHX_STACK_SHARED (a column of a block-wide shared-memory array)
 * or PHX_STACK_REGISTER (the top entry in a register, the older ones in
 * local memory, a pop loading the next entry ahead of use). Same hits in
 * every placement. Batches take LOCAL or
 * SHARED (phx_batch_set_config). */
#define PHX_STACK_LOCAL 0u
#define PHX_STACK_SHARED 1u
#define PHX_STACK_REGISTER 2u
int32_t phx_tracer_set_stack(phx_tracer tr, uint32_t place);
/* How ray-buffer walks (phx_trace_rays) are scheduled: PHX_WALK_THREAD, one
 * thread per ray (the default); PHX_WALK_FETCH, persistent warps whose idle
 * lanes take the next rays from a counter between rounds of 16 visits. Each
 * ray is walked in the same order either way: the same hits. */
#define PHX_WALK_THREAD 0u
#define PHX_WALK_FETCH 1u
/* PHX_WALK_SORTED: PHX_WALK_FETCH over the rays in the order of a stable
 * radix sort by (direction octant, Morton code of the origin), each hit
 * still written at its ray's index. */
#define PHX_WALK_SORTED 2u
/* PHX_WALK_WIDE: persistent warps over a 4-wide tree collapsed on the
 * device from the binary tree (the LBVH or the SAH tree; its boxes and leaf
 * ranges unchanged), at about half the steps a ray, four slab tests a step.
 * The wide tree is made when first walked after a build, refit or tree
 * switch (waits). Closest hits equal the binary walk's but for the face
 * named at a tie (two faces at one t); any-hit rays report the same
 * hit-or-miss. Single-instance scenes. */
#define PHX_WALK_WIDE 3u
/* PHX_WALK_WIDE_THREAD: the same walk of the wide tree, a thread per ray. */
#define PHX_WALK_WIDE_THREAD 4u
int32_t phx_tracer_set_walk(phx_tracer tr, uint32_t mode);
/* Which tree the tracer walks. PHX_TREE_LBVH (the default): the device LBVH
 * (Morton codes, stable radix sort, Karras, leaf packing; 0.6 ms at 1.3 M
 * faces). PHX_TREE_SAH: the binned SAH tree phiray's own tracer builds
 * (src/bvh/sah.rs:85-189, forest.rs:49), node for node, built on the device
 * by phx_bvh_build_sah — fewer node steps and triangle tests a ray, a
 * longer build (1.3 M faces: ~9 ms against 0.5 ms). Closest hits do not
 * depend on the tree (a tie between two
 * faces at the same t aside). Rebuilds the tree now over the current
 * vertices (waits); the image starts over; a repose then refits or rebuilds
 * the same kind. Single-instance scenes (scenes of instances keep LBVH mesh
 * trees: PHX_ERR_INVALID). */
#define PHX_TREE_LBVH 0u
#define PHX_TREE_SAH 1u
int32_t phx_tracer_set_tree(phx_tracer tr, uint32_t tree);
/* The autotuner over trees: builds each (timed, after an untimed build), traces `spp` samples of
 * `cam` on it (timed, after a warm-up trace) and keeps the one with the lower
 * build + frames x trace time — the SAH tree where the trace time of the
 * frames to come outweighs its build. ms (4 floats, may be NULL): LBVH build,
 * LBVH trace, SAH build, SAH trace. Waits; the image is overwritten. */
int32_t phx_tracer_autotune_tree(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t spp,
                                 uint32_t frames, uint32_t* chosen, float* ms);
/* Tracer::set_samples: the sample target `sample` stops at (32 until set,
 * Tracer::SAMPLE_COUNT, src/trace/mod.rs:129). */
int32_t phx_tracer_set_samples(phx_tracer tr, uint32_t samples);
/* Tracer::sample / sample_in (src/trace/sample.rs:94-249): one more sample
 * of `cam` at w x h — frame 0 on a new view, frame + 1 on the same one —
 * in `slices` dispatches, polling `*cancel` (host memory, may be NULL)
 * between them (PHX_ERR_CANCELLED: the sample is abandoned and the next
 * starts over). *frame = the frame traced, *done = 1 once the target is
 * reached (no work is done then). */
int32_t phx_tracer_sample(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t slices,
                          const volatile int32_t* cancel, uint32_t* frame, int32_t* done);
/* Tracer::render's loop as one launch: frames [first, first + spp) of `cam`
 * into the image, each pixel's samples taken in order inside the kernel —
 * the same sums as spp calls of sample. Stream-ordered, no wait. */
int32_t phx_tracer_trace(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first, uint32_t spp);
/* phx_tracer_trace over rows [row0, row0 + rows) of the w x h frame only: the
 * other rows' planes are left as they are. For a frame split across GPUs by
 * rows (each rank traces its rows, then the finished rows are gathered to
 * the presenting rank: phx_tracer_copy_rows). Not with adaptive sampling. */
int32_t phx_tracer_trace_rows(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                              uint32_t spp, uint32_t row0, uint32_t rows);
/* PHX_ROW_WORDS words a pixel of the planes a traced row carries (packed,
 * linear sums, shown, albedo, normal, depth, overlay, coverage, film,
 * outline, sample count, missed — read.rs:37-56): copies rows [row0,
 * row0 + rows) of them between the image and `packed` (DEVICE, plane by
 * plane, PHX_ROW_WORDS * rows * w words), into the image when into_image.
 * Stream-ordered. */
#define PHX_ROW_WORDS 22u
int32_t phx_tracer_copy_rows(phx_tracer tr, uint32_t row0, uint32_t rows, uint32_t* packed, int32_t into_image);
/* Tracer::set_adaptive (src/trace/mod.rs:235-240): Adaptive Sampling as
 * [threshold, min samples, step, on], stamped on every frame this tracer
 * traces in place of the camera's own adapt field (sample.rs:119). With it
 * on, a frame's samples skip the pixels that have settled: at the end of a
 * sample that is a step boundary past the minimum the convergence check of
 * adapt.wgsl runs (full vs half image), then the dilation and the
 * open-pixel list (gather.wgsl) the next samples trace. The image planes
 * are phiray's (half image 26n, flags 29n/30n, list 32n, its length at 34n).
 * A change of setting starts the next sample over. Adaptive frames run on
 * the megakernel forms and whole (no pixel slices); batches refuse them. */
int32_t phx_tracer_set_adaptive(phx_tracer tr, const float adapt[4]);
/* Tracer::show (src/trace/read.rs:182-216, show.wgsl): `count` linear rgb
 * triples (host, row 0 first; missing pixels read as 0) become the image's
 * sums, scaled by the samples each pixel took, and the display step of
 * emit runs over them (shown planes and packed pixels), so a composited
 * image is shown through the same view transform. PHX_ERR_INVALID before
 * any frame was traced. Waits. */
int32_t phx_tracer_show(phx_tracer tr, const float* linear, uint64_t count);
/* Tracer::unconverged (src/trace/mod.rs:224-233): the number of pixels not
 * yet settled after the last sample's tail; PHX_ERR_INVALID when adaptive
 * sampling is off. Bounded wait. */
int32_t phx_tracer_unconverged(phx_tracer tr, uint32_t* count, uint32_t timeout_ms);
/* Tracer::pixels / radiance / ... (read.rs:241-327): `count` words of the
 * image buffer from word `offset` (plane p starts at p * w * h) into host
 * memory; bounded wait. */
int32_t phx_tracer_read(phx_tracer tr, uint64_t offset, uint32_t* dst, uint64_t count, uint32_t timeout_ms);
/* Device pointer and count of the tracer's own vertex array (x, y, z, 1):
 * a skinning kernel can write a new pose straight into it before
 * phx_tracer_repose_device(tr, that pointer, ...), which then copies nothing. */
int32_t phx_tracer_verts(phx_tracer tr, float** verts, uint32_t* nverts);
/* Device pointer and size (words) of the image buffer. */
int32_t phx_tracer_image(phx_tracer tr, uint32_t** px, uint64_t* words);
/* Tracer::denoise / denoise_shown (read.rs:73-119) over the image. */
int32_t phx_tracer_denoise(phx_tracer tr, int32_t keep);
/* Tracer::time (sample.rs:253-255): GPU ms of the last sample/trace call,
 * and the rays it traced (closest-hit and shadow). Waits for it. */
int32_t phx_tracer_time(phx_tracer tr, float* gpu_ms, uint64_t* rays);
/* Tracer::repose on the device (pose.rs:77-100, with the GPU frame path of
 * jobs.md:22): new vertex positions (DEVICE, nverts x 4 f32), face boxes,
 * then an LBVH refit (rebuild = 0) or rebuild (rebuild = 1). */
int32_t phx_tracer_repose_device(phx_tracer tr, const float* verts, int32_t rebuild);
/* The primary ray of frame `frame` per pixel (shade.wgsl:66-95, first
 * trace): hit face id (0xFFFFFFFF for none) and t, into DEVICE arrays of
 * w*h. For hit-id parity checks. */
int32_t phx_tracer_primary(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t frame,
                           uint32_t* ids, float* ts);
/* Closest-hit (any_hit 0) or any-hit (1) walk of `n` rays from DEVICE
 * arrays: rays[2i] = (origin.xyz, tmax), rays[2i+1] = (dir.xyz, 0);
 * hits[i] = (t, face id bits, u, v) with face 0xFFFFFFFF for a miss. */
int32_t phx_trace_rays(phx_tracer tr, const float* rays, uint32_t n, float* hits, int32_t any_hit);
/* The same walks, counted: counts = {rays, inner-node steps, triangle
 * tests} — the work the walk's algorithmic bytes are computed from (one
 * 64-byte node record a step, one 48-byte triangle a test). Waits. */
int32_t phx_trace_rays_stats(phx_tracer tr, const float* rays, uint32_t n, float* hits, int32_t any_hit,
                             uint64_t counts[3]);
/* phx_tracer_trace, counted the same way (rays, steps, tests). Waits. */
int32_t phx_tracer_trace_stats(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                               uint32_t spp, uint64_t counts[3]);
/* The incoherent secondary rays of a frame: for each pixel's primary hit, one
 * cosine-sampled diffuse ray (integrate.wgsl:6-11 cosine_dir) from the
 * lifted hit point, drawn from that pixel's sample stream; written to a
 * DEVICE ray buffer (format of phx_trace_rays, w*h rays; a pixel whose
 * primary ray missed gets a ray with tmax 0). */
int32_t phx_tracer_secondary_rays(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t frame,
                                  float* rays);

/* ---- BF16 tensor-core engine (learned denoiser; no reference counterpart:
 * phiray has no learned denoiser, docs/reconstruct.md:61) ---- */
/* D (fp32 M x N, row-major) = A (bf16 M x K, row-major) x B^T (bf16 N x K,
 * row-major), on tcgen05 tensor cores with the accumulator in TMEM.
 * M % 128 == 0, K % 64 == 0, N in {32, 64, 96, 128, 160}. Device pointers. */
int32_t phx_gemm_bf16(phx_ctx ctx, const void* A, const void* B, float* D, uint32_t M, uint32_t N, uint32_t K);

/* ---- Learned denoiser layers (no reference counterpart). Activations are
 * NHWC bf16 with a pixel pitch and a channel offset (both multiples of 8
 * elements), so a layer reads or writes one channel range of a wider buffer.
 * 3x3 weights are [cout][Kp] bf16 with k = (3 ty + tx) cin + ci, zero from
 * K = 9 cin up to Kp (a multiple of 64). All pointers are device pointers;
 * every call is stream-ordered on the context's stream. ---- */

/* Y[., yo + co] = act(conv3x3(X[., xo + ci]) + bias), stride 1, zero padding 1,
 * cout (one launch's tile) in {32, 64, 96, 128, 160}; relu selects ReLU,
 * out_f32 writes fp32 instead of bf16. */
int32_t phx_nn_conv_fwd(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* W, int32_t Kp,
                        const float* bias, void* Y, int32_t ys, int32_t yo, int32_t cout, int32_t B, int32_t H,
                        int32_t Wd, int32_t relu, int32_t out_f32);
/* The network's head (32 outputs, no ReLU) fused with phx_nn_kpn's forward:
 * out and err exactly as phx_nn_conv_fwd (out_f32) followed by phx_nn_kpn,
 * without writing the logits. */
int32_t phx_nn_conv_kpn(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* W, int32_t Kp,
                        const float* bias, const float* irr, const float* alb, int32_t B, int32_t Hp, int32_t Wp,
                        int32_t h, int32_t w, float* out, float* err);
/* dWt[k][co] += sum over pixels of im2col(X)[p][k] dY[p][dyo + co]; dWt is
 * [Kp][cout] fp32 and must be zeroed by the caller. */
int32_t phx_nn_conv_wgrad(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* dY,
                          int32_t dys, int32_t dyo, int32_t cout, float* dWt, int32_t Kp, int32_t B, int32_t H,
                          int32_t Wd);
/* db[c] += sum over the P pixels of dY[p][dyo + c] (C <= 256). */
int32_t phx_nn_bias_grad(phx_ctx ctx, const void* dY, int32_t dys, int32_t dyo, int32_t C, int32_t P, float* db);
/* dY[p][c] = 0 where Y[p][c] <= 0 (ReLU's gradient through its output). */
int32_t phx_nn_relu_bwd(phx_ctx ctx, const void* Y, int32_t ys, int32_t yo, void* dY, int32_t dys, int32_t dyo,
                        int32_t C, int32_t P);
/* 2x2 average pooling of (B, H, W) into a contiguous (B, H/2, W/2, C). */
int32_t phx_nn_pool_fwd(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t C, int32_t B, int32_t H, int32_t W,
                        void* Y);
/* Its gradient, ADDED into dX (B, H, W; pitch dxs, offset dxo). */
int32_t phx_nn_pool_bwd(phx_ctx ctx, const void* dY, int32_t C, int32_t B, int32_t H, int32_t W, void* dX, int32_t dxs,
                        int32_t dxo);
/* Nearest 2x upsampling of a contiguous (B, H/2, W/2, C) into (B, H, W). */
int32_t phx_nn_up_fwd(phx_ctx ctx, const void* X, int32_t C, int32_t B, int32_t H, int32_t W, void* Y, int32_t ys,
                      int32_t yo);
/* Its gradient: dX (B, H/2, W/2, C contiguous) = sum over each 2x2 block. */
int32_t phx_nn_up_bwd(phx_ctx ctx, const void* dY, int32_t dys, int32_t dyo, int32_t C, int32_t B, int32_t H, int32_t W,
                      void* dX);
/* W2[ci][(8 - tap) cout + co] = W[co][tap cin + ci]: the weights whose 3x3
 * convolution of dY is the data gradient. W2 is [cin][Kp2]. */
int32_t phx_nn_flip(phx_ctx ctx, const void* W, int32_t cout, int32_t cin, int32_t Kp, void* W2, int32_t Kp2);
/* Per-pixel 5x5 kernels (softmax of logits 0..24, pitch 32 fp32) over the
 * demodulated radiance irr (fp32 x 3), clamped to the valid h x w corner of
 * the padded Hp x Wp images, remodulated by alb: out = alb * sum w irr.
 * err = exp(logit 25) - 1e-3 (the error estimate). With ref: *loss += mean
 * relative squared error (x - r)^2 / (r^2 + 0.01), and dlogits (bf16 pitch
 * 32) = its gradient plus err_weight times that of the error head's squared
 * log error. out, err, ref, dlogits, loss may be NULL. */
int32_t phx_nn_kpn(phx_ctx ctx, const float* logits, const float* irr, const float* alb, const float* ref, int32_t B,
                   int32_t Hp, int32_t Wp, int32_t h, int32_t w, float* out, float* err, void* dlogits, float* loss,
                   float err_weight);
/* Adam (bias-corrected, step >= 1) on a [rows][Kp] fp32 matrix whose first K
 * columns are live; the gradient is [Kp][rows] when g_transposed, else
 * [rows][Kp]. wb (nullable) receives the bf16 copy. */
int32_t phx_nn_adam(phx_ctx ctx, float* w, const float* g, float* m, float* v, void* wb, int32_t rows, int32_t Kp,
                    int32_t K, int32_t g_transposed, float lr, float b1, float b2, float eps, int32_t step);
/* Network inputs from a traced px image (w x h) into padded Hp x Wp planes:
 * feat (16 bf16 channels), irr and alb (fp32 x 3). half (nullable): a
 * phx_nn_snapshot of the same image taken part way through its samples,
 * from which the pixels' own sample spread is read. */
int32_t phx_nn_features(phx_ctx ctx, const uint32_t* px, const float* half, int32_t w, int32_t h, int32_t Hp,
                        int32_t Wp, void* feat, float* irr, float* alb);
/* The a-trous Denoise's first-round firefly clamp (denoise.wgsl:47-134) on B
 * padded Hp x Wp images of fp32 x 3 irradiance, inside the h x w image: a
 * pixel brighter in luma than 1.5 x its brightest 8-neighbour + 0.05 takes
 * their mean. out must not alias irr. */
int32_t phx_nn_firefly(phx_ctx ctx, const float* irr, float* out, int32_t B, int32_t Hp, int32_t Wp, int32_t h,
                       int32_t w);
/* A snapshot of a px image's linear sums and met-sample counts (w * h x 4
 * floats, device): the `half` input of phx_nn_features. */
int32_t phx_nn_snapshot(phx_ctx ctx, const uint32_t* px, uint32_t w, uint32_t h, float* snap);
/* Per tile x tile block: mean error estimate into tile_err and the count of
 * tiles above threshold into *fallback (device); every pixel of a tile within
 * the threshold gets `out` written into the px planes (sums unless keep,
 * shown, packed), the others keep what the a-trous Denoise wrote. */
int32_t phx_nn_compose(phx_ctx ctx, uint32_t* px, int32_t w, int32_t h, int32_t Wp, const float* out, const float* err,
                       int32_t tile, float threshold, int32_t keep, float exposure, float gamma, float* tile_err,
                       uint32_t* fallback);

/* ---- The learned denoiser: a kernel-predicting U-Net (5 levels of 32, 64,
 * 96, 128, 160 channels, two 3x3 convolutions per level each way, 5x5
 * per-pixel kernels) trained and run on the device. ---- */
typedef struct phx_unet_s* phx_unet;
/* A network with He-initialised weights drawn from `seed`. */
int32_t phx_unet_create(phx_ctx ctx, uint64_t seed, phx_unet* out);
int32_t phx_unet_destroy(phx_unet net);
/* Parameters in the blob layout: per layer W [cout][9 cin] then b [cout]. */
int32_t phx_unet_param_count(phx_unet net, uint64_t* count);
/* Loads fp32 weights (host) and resets the optimiser. */
int32_t phx_unet_set_params(phx_unet net, const float* params, uint64_t count);
/* which = 0: the weights; 1: the gradients of the last phx_unet_grads. */
int32_t phx_unet_get(phx_unet net, int32_t which, float* dst, uint64_t count);
/* Forward over B padded images Hp x Wp (multiples of 16) of 16-channel
 * features; out / err as phx_nn_kpn (nullable: logits only). */
int32_t phx_unet_forward(phx_unet net, const void* feat, const float* irr, const float* alb, int32_t B, int32_t Hp,
                         int32_t Wp, int32_t h, int32_t w, float* out, float* err);
/* Forward, loss against ref (added to *loss, device) and all gradients. */
int32_t phx_unet_grads(phx_unet net, const void* feat, const float* irr, const float* alb, const float* ref, int32_t B,
                       int32_t Hp, int32_t Wp, int32_t h, int32_t w, float err_weight, float* loss);
/* One Adam step (b1 0.9, b2 0.999, eps 1e-8) with the last gradients. */
int32_t phx_unet_adam(phx_unet net, float lr);
/* Every layer's gradients as one device array of *count fp32 (per layer the
 * weight gradient [Kp][cout], Kp = 9 cin rounded up to 64, then the bias
 * gradient [cout], each starting at a multiple of 64 floats; the padding is
 * zero). Data-parallel training reduces this one array across ranks between
 * phx_unet_grads and phx_unet_adam (an all-reduce average), so every rank
 * takes the same Adam step. No reference counterpart: phiray trains no
 * network. */
int32_t phx_unet_grad_arena(phx_unet net, float** grads, uint64_t* count);
/* phx_unet_grads then phx_unet_adam. */
int32_t phx_unet_train_step(phx_unet net, const void* feat, const float* irr, const float* alb, const float* ref,
                            int32_t B, int32_t Hp, int32_t Wp, int32_t h, int32_t w, float err_weight, float lr,
                            float* loss);
/* Device pointer of the last forward's head output ([B][Hp][Wp][32] fp32). */
int32_t phx_unet_logits(phx_unet net, float** logits);
/* Whether phx_unet_denoise_px's predicted kernels filter the irradiance
 * after phx_nn_firefly (on) or as it is (0, the default). */
int32_t phx_unet_set_clamp(phx_unet net, int32_t on);
/* Test-time flip average of phx_unet_denoise_px / phx_tracer_denoise_learned:
 * the filtered image and its error estimate are the mean over `images`
 * network passes, the frame (1, the default), also mirrored in x (2), and
 * mirrored in y and in both (4); each mirrored pass's kernels filter its
 * own mirrored irradiance. Costs one network pass an image. */
int32_t phx_unet_set_flips(phx_unet net, int32_t images);
/* Denoises a traced px image in place (`half`: nullable snapshot, as
 * phx_nn_features): features, network (its kernels filtering the
 * firefly-clamped irradiance if phx_unet_set_clamp turned that on), the a-trous
 * Denoise (phx_denoise, strength 64/8/40/7), then the learned result on every
 * tile x tile block whose mean error estimate is <= threshold. With
 * `fallback` non-NULL, waits and returns the number of tiles that kept the
 * a-trous result. */
int32_t phx_unet_denoise_px(phx_unet net, uint32_t* px, const float* half, uint32_t w, uint32_t h,
                            const float view[4], int32_t tile, float threshold, int32_t keep, uint32_t* fallback);
/* phx_nn_snapshot of the tracer's image as it is now (take it half way
 * through a frame's samples and pass it to phx_tracer_denoise_learned). */
int32_t phx_tracer_snapshot(phx_tracer tr, float* snap);
/* Tracer::denoise with the learned denoiser (phx_unet_denoise_px on the
 * tracer's image, `half` (nullable) and the last camera's view); nothing
 * traced: no-op. */
int32_t phx_tracer_denoise_learned(phx_tracer tr, phx_unet net, const float* half, int32_t tile, float threshold,
                                   int32_t keep, uint32_t* fallback);

/* ---- Batched serving: many tracers' frames in one persistent launch (no
 * reference counterpart; phiber renders one Tracer per view). ---- */
typedef struct phx_batch_s* phx_batch;
/* PHX_BATCH_PERSISTENT: one launch whose warps take 32-pixel tiles of every
 * job from one counter (costliest jobs first); PHX_BATCH_PER_SCENE: one
 * launch per job with its tracer's own render kernel. Every job's image is
 * bit for bit its tracer's own phx_tracer_trace. */
#define PHX_BATCH_PERSISTENT 0u
#define PHX_BATCH_PER_SCENE 1u
/* PHX_BATCH_PERSISTENT_DENSE: the persistent launch with registers budgeted
 * for every thread slot of an SM resident (32 a thread; PHX_BATCH_PERSISTENT
 * budgets 1,536 threads, 40 registers). */
#define PHX_BATCH_PERSISTENT_DENSE 2u
int32_t phx_batch_create(phx_ctx ctx, phx_batch* out);
int32_t phx_batch_destroy(phx_batch b);
/* A job: frames [first, first + spp) of `cam` at w x h into tracer tr's image
 * (one job per tracer). The camera is copied. */
int32_t phx_batch_add(phx_batch b, phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                      uint32_t spp, uint32_t* index);
int32_t phx_batch_clear(phx_batch b);
/* Launch form, block size (64, 128, 256) and walk-stack placement
 * (PHX_STACK_LOCAL / PHX_STACK_SHARED) of the persistent kernel. */
int32_t phx_batch_set_config(phx_batch b, uint32_t kind, uint32_t threads, uint32_t stack);
/* Every job's frame, stream-ordered. */
int32_t phx_batch_trace(phx_batch b);
/* The autotuner: times the persistent launch at each block size and stack
 * placement, the dense persistent launch at 128 and 256 threads, and
 * per-scene launches of the megakernel (4 and 16 resident blocks) and of the
 * state machine, on the batch; keeps the fastest. ms (>= 11 floats, may be NULL)
 * gets each configuration's time, *nconfigs their number. Waits. */
int32_t phx_batch_autotune(phx_batch b, uint32_t* kind, uint32_t* threads, uint32_t* stack, float* ms,
                           uint32_t* nconfigs);
/* Records one serving frame as a CUDA graph: per job its face boxes, an LBVH
 * rebuild and a refit each gated by the job's mode word, the tracer's
 * preparation; the batch trace; per job the learned denoiser with the
 * a-trous fallback (net non-NULL; one copy of the network per image shape)
 * or the a-trous Denoise, then a completion time stamp. Runs one frame
 * outside the capture first (sizing every buffer). Tracers of instances or
 * on an SAH tree are refused (PHX_ERR_INVALID): phx_batch_trace takes them. */
int32_t phx_batch_capture(phx_batch b, phx_unet net, float threshold);
/* Replays the captured frame; modes (HOST, one per job): 1 rebuild, 0 refit. */
int32_t phx_batch_replay(phx_batch b, const uint32_t* modes);
/* After a replay: each job's completion time after the frame's start (ns,
 * device clock) and rays traced (both nullable, one per job). Waits. */
int32_t phx_batch_results(phx_batch b, uint64_t* latency_ns, uint64_t* rays);

#ifdef __cplusplus
}
#endif

#endif /* PHIRAY_CUDA_H */
