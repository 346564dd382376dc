// The render kernels of the Rendered-mode tracer (shade.wgsl main and what
// it calls): the megakernel, the persistent state machine, the batched
// persistent launch and the wavefront render, with their launch templates.
// Each render_*.cu file instantiates a share of the kernel forms, so the
// forms compile in parallel; trace.cu holds the host code and calls them
// through the functions declared here.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstring>

#include "shade.cuh"

namespace phx {

using namespace shade;

// One render launch: the scene and frame records and the buffers it writes.
struct RenderLaunch {
    Scene S;
    Frame F;
    f3 sun;
    uint32_t* px;
    uint32_t first, count;
    unsigned long long* counters;
    uint32_t* next;
    int sms;
    cudaStream_t s;
};

// The wavefront render's buffers (see launch_wf).
struct WfBuffers {
    uint32_t nslots;
    uint32_t* words;
    float4* rays;
    float4* hits;
    uint32_t* hinst;
    uint32_t* queues;
    uint32_t* lens;
    uint32_t* host_lens;  // pinned, 3 words
};

constexpr uint32_t WF_SLOTS = 1u << 20;  // path slots of the wavefront render (at most)
// 32-bit words of one wavefront path slot (Path, Sums, phase).
uint32_t wf_slot_words();

// The single-instance render kernels by id: ids 0 and 4-8 (render_flat_a.cu),
// 9-12 (render_flat_b.cu), 13-15 (render_flat_c.cu), 17-19 (render_flat_r.cu),
// 1-3 (render_sm.cu).
int32_t render_flat_a(uint32_t kernel, bool stats, const RenderLaunch& L);
int32_t render_flat_b(uint32_t kernel, bool stats, const RenderLaunch& L);
int32_t render_flat_c(uint32_t kernel, bool stats, const RenderLaunch& L);
int32_t render_flat_r(uint32_t kernel, bool stats, const RenderLaunch& L);
int32_t render_flat_sm(uint32_t kernel, bool stats, const RenderLaunch& L);
// Scenes of instances and frames with the floor grid (render_full.cu).
int32_t render_full(uint32_t kernel, bool stats, const RenderLaunch& L);
// The wavefront render (render_wf.cu).
int32_t render_wavefront(bool full, bool stats, const RenderLaunch& L, const WfBuffers& B);
// The batched persistent launch over a device job table (render_batch.cu):
// `threads` 64, 128 or 256, the walk stacks in shared memory when smem_stack,
// registers for 2048 resident threads an SM when dense (else 1536).
int32_t render_batch(int threads, bool full, bool smem_stack, bool dense, int device, int sms, const void* jobs,
                     uint32_t njobs, uint32_t ntiles, uint32_t* next, cudaStream_t s);
// sizeof the batch kernel's job record.
size_t batch_job_bytes();
// The 4-wide tree collapsed from the tracer's binary records `bin` (wide.cu):
// at most `ninner` 128-byte wide records (0: the root is a leaf, nothing to
// build); jobs_a/jobs_b hold ninner (wide id, record) pairs each, counts 2
// words. Waits on `s` once a level.
int32_t build_wide(const float4* bin, uint32_t ninner, float4* wide, uint2* jobs_a, uint2* jobs_b, uint32_t* counts,
                   cudaStream_t s, uint32_t* nodes_out, uint32_t* levels_out);
// Walks of n rays over the wide tree: persistent warps (next: one word of
// scratch) or, with next null, a thread a ray (counters: rays, steps, tests,
// or null).
int32_t launch_rays_wide(const Scene& S, const float4* wide, const float* rays, uint32_t n, float* hits, bool any,
                         unsigned long long* counters, uint32_t* next, int sms, cudaStream_t s);

namespace {

// ---- the sample kernel (shade.wgsl main) ----

struct Sums {
    f3 lin, grid, alb, nrm;
    f3 half;  // Adaptive Sampling's half image: every odd sample at double weight
    float cov, film, gone, dep;
    uint32_t count, outline;
};

__device__ __forceinline__ float srgb_to_linear1(float c) {
    return c <= 0.04045f ? c / 12.92f : pm_pow((c + 0.055f) / 1.055f, 2.4f);
}

__device__ __forceinline__ f3 env_at(const Frame& F) { return F.env; }

// direct (integrate.wgsl:66-85): every light with its shadow ray.
template <int STATS>
__device__ __noinline__ f3 direct(const Scene& S, const Frame& F, const Surf& s, uint32_t& seed, bool with_env,
                                  f3 sun, Count& cnt) {
    const bool rig = uses_rig(F);
    f3 sum = rig ? rig_fill(F, s) : mk(0.0f);
    for (uint32_t k = 0; k < 4u; k++) {
        Shadowed q = unshadowed();
        if (k == 0u) {
            q = rig ? rig_query(F, 0u, s, seed, sun) : lamp_query(F, s, seed);
        } else if (k == 1u) {
            if (rig) q = rig_query(F, 1u, s, seed, sun);
        } else if (k == 2u) {
            q = glow_query<STATS>(S, s, seed);
        }
        // k == 3: env_query needs an environment image's table (env_cdf),
        // which the host refuses; it returns unshadowed without a draw.
        if (maxc(q.c) > 0.0f) {
            const float vis = trace<STATS>(S, s.pos, q.dir, q.dist, true, cnt).tri != NONE ? 0.0f : 1.0f;
            sum += q.c * vis;
        }
    }
    return sum;
}

// glow_mis (integrate.wgsl:15-23).
template <int M>
__device__ __forceinline__ f3 glow_mis(const Scene& S, const Geo& g, f3 emit, const Hit& h, f3 from_n, f3 dir) {
    const float chance = lamp_chance<M>(S, h.tri, (M & MODE_FULL) ? h.inst : 0u);
    if (chance <= 0.0f) return emit;
    const f3 cr = cross(g.b - g.a, g.c - g.a);
    const float pl = chance * h.t * h.t / fmaxf(0.5f * length(cr) * fabsf(dot(normalize(cr), dir)), 1e-8f);
    const float pb = fmaxf(dot(from_n, dir), 0.0f) / PI;
    return emit * pb * pb / fmaxf(pb * pb + pl * pl, 1e-12f);
}

// indirect (integrate.wgsl:111-230) with no environment image.
template <int STATS>
__device__ __forceinline__ f3 indirect(const Scene& S, const Frame& F, f3 pos, f3 n, uint32_t& seed, bool bounce,
                                       f3 sun, Count& cnt) {
    const bool lit = dot(F.env, F.env) > 0.0f;
    if (S.lamp_count == 0u && !lit) {
        const f3 dir = cosine_dir(n, seed);
        // env_at(dir) * mix(0.25, 1, visible(pos, dir, ao)): with a black
        // world the product is zero whatever the shadow ray finds, so the
        // ray is only traced when the world has some colour.
        if (F.env.x == 0.0f && F.env.y == 0.0f && F.env.z == 0.0f) return mk(0.0f);
        const float vis = trace<STATS>(S, pos, dir, F.ao, true, cnt).tri != NONE ? 0.0f : 1.0f;
        return env_at(F) * mixf(0.25f, 1.0f, vis);
    }
    const uint32_t depth = bounce ? (F.bounces != 0u ? F.bounces : 1u) : 1u;
    f3 acc = mk(0.0f), thr = mk(1.0f), org = pos, nrm = n;
    float min_pdf = 3.0e38f;
    bool through = false;
    f3 dir = mk(0.0f, 0.0f, 1.0f);
    float pb = 1.0f;
    for (uint32_t b = 0; b < depth; b++) {
        if (!through) {
            dir = cosine_dir(nrm, seed);
            pb = fmaxf(dot(nrm, dir), 0.0f) / PI;
        }
        through = false;
        min_pdf = fminf(min_pdf, pb);
        const Hit h = trace<STATS>(S, org, dir, INF, false, cnt);
        if (h.tri == NONE) {
            acc += thr * env_at(F) * 1.0f;
            break;
        }
        if (!bounce) break;
        const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
        const Mat t = mat_at(S, g.mat);
        const f3 ng0 = normalize(cross(g.b - g.a, g.c - g.a));
        const f3 ng = dot(ng0, dir) < 0.0f ? ng0 : -ng0;
        const f3 hit = org + dir * h.t + ng * (F.eps + h.t * 1e-5f);
        const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
        const float rough = fmaxf(t.rough, glossy_floor());
        const f3 fd = dielectric_f0(t.ior);
        const float metal = t.metal;
        const float tw = t.trans * (1.0f - t.metal);
        f3 albedo = base * (1.0f - t.metal) * (1.0f - tw);
        if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxf(dot(ng, -dir), 1e-4f));
        acc += thr * glow_mis<STATS>(S, g, t.emit, h, nrm, dir);
        const float near = (!lit && h.t <= F.ao) ? 0.25f : 1.0f;
        const Surf s = plain_surf(hit, ng, -dir, albedo, vmix(fd, base, metal), rough);
        acc += thr * direct<STATS>(S, F, s, seed, true, sun, cnt) * near;
        if (tw > 0.0f && rnd(seed) < tw) {
            thr *= mk(sqrtf(base.x), sqrtf(base.y), sqrtf(base.z));
            const f3 at = org + dir * h.t;
            org = at - ng * through_lift(F, at, h.t);
            through = true;
            continue;
        }
        thr *= albedo;
        if (b + 1u < depth) {
            const float keep = clampf(maxc(thr), 0.0f, 0.95f);
            if (keep < 1e-4f || rnd(seed) > keep) break;
            thr = thr / keep;
        }
        org = hit;
        nrm = ng;
    }
    return acc;
}

// bounce_light (integrate.wgsl:236-250).
template <int STATS>
__device__ __forceinline__ f3 bounce_light(const Scene& S, const Frame& F, const Hit& h, f3 org, f3 d,
                                           uint32_t& seed, f3 sun, Count& cnt) {
    const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
    const Mat t = mat_at(S, g.mat);
    const f3 ng0 = normalize(cross(g.b - g.a, g.c - g.a));
    const f3 ng = dot(ng0, d) < 0.0f ? ng0 : -ng0;
    const f3 pos = org + d * h.t + ng * (F.eps + h.t * 1e-5f);
    const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
    const float rough = fmaxf(t.rough, glossy_floor());
    const f3 fd = dielectric_f0(t.ior);
    f3 albedo = base * (1.0f - t.metal);
    if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxf(dot(ng, -d), 1e-4f));
    const Surf s = plain_surf(pos, ng, -d, albedo, vmix(fd, base, t.metal), rough);
    return direct<STATS>(S, F, s, seed, false, sun, cnt) + s.albedo * env_at(F) * 0.8f + t.emit;
}

__device__ __forceinline__ f3 clamp_light(f3 l, float limit) {
    const float m = fmaxf(l.x, fmaxf(l.y, l.z));
    if (limit <= 0.0f || m <= limit) return l;
    return l * (limit / m);
}

struct CamRay {
    f3 o, d;
};

__device__ __forceinline__ CamRay camera_ray(const Frame& F, uint32_t i, uint32_t& seed) {
    const float su = ((float)(i % F.w) + 0.5f) / (float)F.w - 0.5f;
    const float sv = ((float)(i / F.w) + 0.5f) / (float)F.h - 0.5f;
    const float jox = rnd(seed) - 0.5f;
    const float joy = rnd(seed) - 0.5f;
    const float jx = jox / (float)F.w;
    const float jy = joy / (float)F.h;
    const float vx = (su + jx - F.pan_x) / F.scale;
    const float vy = -((sv + jy) / F.aspect - F.pan_y) / F.scale;
    CamRay r;
    if (F.persp != 0u) {
        r.o = F.pivot + F.back * (F.dist / F.units);
        r.d = normalize(F.right * vx + F.up * vy - F.back * F.dist);
    } else {
        r.o = F.pivot + (F.right * vx + F.up * vy + F.back * 1.0e4f) / F.units;
        r.d = -F.back;
    }
    return r;
}

// One sample of pixel i (shade.wgsl:41-373) added into `acc`.
template <int STATS>
__device__ void sample(const Scene& S, const Frame& F, uint32_t i, uint32_t frame, f3 sun, Sums& acc,
                       Count& cnt) {
    uint32_t seed = hash(i * 9781u + frame * 6271u + 1u);
    const CamRay cr = camera_ray(F, i, seed);
    f3 o = cr.o, d = cr.d;
    acc.outline = 0;
    f3 col = mk(0.0f), thr = mk(1.0f);
    const uint32_t see_through = 8u, through = 8u;
    const bool glossy_on = true, diffuse_on = true;
    uint32_t n_see = 0, n_through = 0;
    const uint32_t passes = see_through + through + 1u;
    for (uint32_t bounce = 0; bounce < passes; bounce++) {
        const Hit h = trace<STATS>(S, o, d, INF, false, cnt);
        if (h.tri == NONE) {
            if (bounce == 0u) {
                const float across = (float)(i % F.w) / fmaxf((float)F.w * 0.5f, 1.0f);
                const float lift = F.sky[3] * (1.0f - clampf(across, 0.0f, 1.0f));
                const f3 sky = mk(F.sky[0] + lift, F.sky[1] + lift, F.sky[2] + lift);
                acc.alb += mk(srgb_to_linear1(sky.x), srgb_to_linear1(sky.y), srgb_to_linear1(sky.z));
                acc.nrm += -d;
                acc.dep += -1.0f;
                acc.gone += 1.0f;
                acc.count += 1u;
                acc.film += 1.0f;
                acc.lin += mk(0.0f);
                if (F.adapt_on && (frame & 1u)) acc.half = acc.half + mk(0.0f) * 2.0f;
                if ((STATS & MODE_FULL) && F.grid > 0.0f) {
                    const Over g = grid_over(F, o, d, INF);
                    acc.grid += sky * (1.0f - g.a) + g.c;
                } else {
                    acc.grid += sky * (1.0f - 0.0f) + mk(0.0f);
                }
                acc.cov += 1.0f;
                return;
            }
            col += thr * env_at(F);
            break;
        }
        if (bounce == 0u) {
            acc.outline = ((STATS & MODE_FULL) ? h.inst : 0u) + 1u;  // outline_store(i, h.inst + 1)
            // emit's overlay term grid_over(o0, d0, first_t) is a function of
            // the first ray and hit alone: added once per sample here, where
            // they are at hand, instead of at emit (util.wgsl:101-145)
            if ((STATS & MODE_FULL) && F.grid > 0.0f) {
                const Over gr = grid_over(F, o, d, h.t);
                acc.grid += gr.c;
                acc.cov += gr.a;
            }
        }
        const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
        const Mat t = mat_at(S, g.mat);
        const float w = 1.0f - h.u - h.v;
        const f3 hit = o + d * h.t;
        const f3 ngw = normalize(cross(g.b - g.a, g.c - g.a));
        const f3 ng0 = g.mirror ? -ngw : ngw;  // world_ng (layout.wgsl:97-101)
        const bool front = dot(ng0, d) < 0.0f;
        const f3 ng = front ? ng0 : -ng0;
        f3 n = g.na * w + g.nb * h.u + g.nc * h.v;
        n = dot(n, n) > 1e-12f ? normalize(n) * (front ? 1.0f : -1.0f) : ng;
        if (dot(n, -d) < 0.0f) n = ng;
        const f3 off = ng * hit_lift(F, h.t);
        const f3 past = ng * through_lift(F, hit, h.t);
        const f3 pos = hit + off;
        const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
        const float alpha = t.color.w;
        const float rough = t.rough;
        const float metal = t.metal;
        const f3 emit = t.emit;
        if (bounce == 0u) {
            acc.alb += base;
            acc.nrm += n;
            acc.dep += h.t;
        }
        if (rnd(seed) >= alpha) {
            n_see++;
            if (n_see > see_through) break;
            o = hit - past;
            continue;
        }
        col += thr * emit;
        const float bleed = scatter_bleed(t.sss, t.sss_radius);
        const f3 fd = dielectric_f0(t.ior);
        f3 diffuse = base * (1.0f - metal);
        if (maxc(diffuse) > 0.0f) diffuse *= under_layer_real(t.ior, fmaxf(rough, 0.04f), fmaxf(dot(n, -d), 1e-4f));
        const Surf s{pos,   n,      -d,        diffuse,         vmix(fd, base, metal), fmaxf(rough, 0.04f),
                     bleed, scatter_tint(t.sss_radius), t.sheen, t.sheen_rough,    t.sheen_tint,
                     t.coat, t.coat_rough, t.ior, 1.0f - metal};
        const float opaque = 1.0f - t.trans * (1.0f - metal);
        f3 c = mk(0.0f);
        if (opaque > 0.0f) c = direct<STATS>(S, F, s, seed, true, sun, cnt) * opaque;
        if (opaque < 1.0f) {
            const Surf shine{pos, n, -d, mk(0.0f), s.f0, s.rough, 0.0f, mk(1.0f), 0.0f, t.sheen_rough,
                             t.sheen_tint, t.coat, t.coat_rough, s.eta, s.dielectric};
            c += direct<STATS>(S, F, shine, seed, true, sun, cnt) * (1.0f - opaque);
        }
        c = clamp_light(c, F.limit_d);
        f3 bounced = mk(0.0f);
        const f3 diffuse_weight = vmix(s.albedo, s.albedo * s.sss_tint, bleed) * opaque;
        const f3 lw = mk(0.2126f, 0.7152f, 0.0722f);
        const float ndv = fmaxf(dot(n, -d), 1e-4f);
        const f3 gloss_guess = s.f0 + (mk(1.0f) - s.f0) * pm_pow(1.0f - ndv, 5.0f);
        const float pd = dot(vmax(diffuse_weight, mk(0.0f)), lw);
        const float pg = glossy_on ? dot(gloss_guess, lw) : 0.0f;
        float p_diffuse = pd + pg > 0.0f ? pd / (pd + pg) : 1.0f;
        if (pd > 0.0f && pg > 0.0f) p_diffuse = clampf(p_diffuse, 0.15f, 0.85f);
        const bool take_diffuse = rnd(seed) < p_diffuse;
        if (take_diffuse && pd > 0.0f)
            bounced += diffuse_weight * indirect<STATS>(S, F, pos, n, seed, diffuse_on, sun, cnt) / p_diffuse;
        const f3 v = -d;
        const f3 tx = normalize(onb(n, 1.0f, 0.0f));
        const f3 ty = cross(n, tx);
        const float ggx_a = s.rough * s.rough;
        const f3 wi_local = mk(dot(v, tx), dot(v, ty), dot(v, n));
        const float r1 = rnd(seed);
        const float r2 = rnd(seed);
        const f3 h_local = ggx_sample_vndf(wi_local, ggx_a, r1, r2);
        const f3 hw = normalize(tx * h_local.x + ty * h_local.y + n * h_local.z);
        const f3 refl = reflect(d, hw);
        const float cos_hi = fmaxf(dot(hw, v), 0.0f);
        const float cos_no = dot(n, refl);
        const f3 fres = fresnel_of(s, cos_hi);
        if (!take_diffuse && glossy_on && dot(refl, ng) > 0.0f && cos_hi > 0.0f && cos_no > 0.0f) {
            const Hit rh = trace<STATS>(S, pos, refl, INF, false, cnt);
            f3 rc = env_at(F);
            const float wg = 1.0f;
            if (rh.tri != NONE) rc = bounce_light<STATS>(S, F, rh, pos, refl, seed, sun, cnt);
            bounced += fres * rc * ggx_weight(ggx_a * ggx_a, fmaxf(dot(n, v), 1e-4f), cos_no) * wg / (1.0f - p_diffuse);
        }
        c += clamp_light(bounced, F.limit_i);
        col += thr * c;
        const float tw = t.trans * (1.0f - metal);
        if (tw <= 0.0f) break;
        n_through++;
        if (n_through > through) break;
        const float eta = front ? 1.0f / t.ior : t.ior;
        f3 nd = refract(d, n, eta);
        if (dot(nd, nd) < 1e-6f) {
            nd = reflect(d, n);
            o = hit + past;
            thr *= tw;
        } else {
            o = hit - past;
            thr *= mk(sqrtf(base.x), sqrtf(base.y), sqrtf(base.z)) * tw * (mk(1.0f) - fres);
        }
        d = cone_dir(normalize(nd), s.rough * s.rough, seed);
        if (maxc(thr) < 0.01f) break;
    }
    // emit (util.wgsl:101-145); the overlay was added at the first hit.
    acc.gone += 0.0f;
    acc.count += 1u;
    acc.film += 1.0f;
    acc.lin += col;
    // the half image takes the odd samples at double weight (util.wgsl:126-132)
    if (F.adapt_on && (frame & 1u)) acc.half = acc.half + col * 2.0f;
}

__device__ __forceinline__ void ld3(const uint32_t* px, uint32_t base, uint32_t i, f3& v) {
    v = mk(__uint_as_float(px[base + 3 * i]), __uint_as_float(px[base + 3 * i + 1]),
           __uint_as_float(px[base + 3 * i + 2]));
}

__device__ __forceinline__ void st3(uint32_t* px, uint32_t base, uint32_t i, f3 v) {
    px[base + 3 * i] = __float_as_uint(v.x);
    px[base + 3 * i + 1] = __float_as_uint(v.y);
    px[base + 3 * i + 2] = __float_as_uint(v.z);
}

__device__ __forceinline__ void setup(Scene& S, Frame& F) {
    load_info(S);
    if (!(F.ao > 0.0f)) F.ao = S.extent * 0.08f;
    F.eps = S.extent * 1e-5f;
}

// One pixel's samples [F.frame0, F.frame0 + F.spp): its sums read back (or
// started over on frame 0), shade.wgsl's main once per sample, the planes
// written once (util.wgsl's guide/emit over the whole run of samples).
// SYNC: the lanes that entered wait for each other after every sample, so
// each sample's camera ray and first bounces start together (the same sums
// either way: a lane's own samples keep their order).
template <int STATS, bool SYNC = false>
__device__ __forceinline__ void render_px(const Scene& S, const Frame& F, f3 sun, uint32_t* __restrict__ px,
                                          uint32_t i, Count& cnt) {
    const unsigned lanes = __activemask();
    const uint32_t n = F.n;
    Sums acc;
    if (F.frame0 > 0u) {
        ld3(px, 1 * n, i, acc.lin);
        ld3(px, 20 * n, i, acc.grid);
        ld3(px, 7 * n, i, acc.alb);
        ld3(px, 10 * n, i, acc.nrm);
        acc.cov = __uint_as_float(px[23 * n + i]);
        acc.film = __uint_as_float(px[24 * n + i]);
        acc.gone = __uint_as_float(px[33 * n + i]);
        acc.dep = __uint_as_float(px[13 * n + i]);
        acc.count = px[31 * n + i];
    } else {
        acc.lin = acc.grid = acc.alb = acc.nrm = mk(0.0f);
        acc.cov = acc.film = acc.gone = acc.dep = 0.0f;
        acc.count = 0;
        px[29 * n + i] = 0u;
        px[30 * n + i] = 0u;
    }
    // The half image is read whatever the frame: the first odd sample adds
    // to what the plane holds, as util.wgsl's emit does (`keep` is true
    // from frame 1 on, and frame 0 never writes the plane).
    if (F.adapt_on) ld3(px, 26 * n, i, acc.half);
    acc.outline = 0;
    for (uint32_t s = 0; s < F.spp; s++) {
        sample<STATS>(S, F, i, F.frame0 + s, sun, acc, cnt);
        if (SYNC) __syncwarp(lanes);
    }
    st3(px, 1 * n, i, acc.lin);
    st3(px, 20 * n, i, acc.grid);
    st3(px, 7 * n, i, acc.alb);
    st3(px, 10 * n, i, acc.nrm);
    px[23 * n + i] = __float_as_uint(acc.cov);
    px[24 * n + i] = __float_as_uint(acc.film);
    px[33 * n + i] = __float_as_uint(acc.gone);
    px[13 * n + i] = __float_as_uint(acc.dep);
    px[31 * n + i] = acc.count;
    px[25 * n + i] = acc.outline;
    if (F.adapt_on) st3(px, 26 * n, i, acc.half);
    const float kk = (float)acc.count;
    const f3 shown = view_transform_std(acc.lin / fmaxf(kk - acc.gone, 1.0f), F.exposure, F.gamma) *
                         (1.0f - acc.cov / kk) +
                     acc.grid / kk;
    st3(px, 4 * n, i, shown);
    px[i] = pack_rgba(shown, acc.film / kk);
}

// Adds a warp's ray count (and STATS: steps, tests) to counters[0..2].
template <int STATS>
__device__ __forceinline__ void flush_counts(const Count& cnt, unsigned long long* counters) {
    const uint32_t tot = __reduce_add_sync(0xffffffffu, cnt.rays);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(counters, (unsigned long long)tot);
    if (STATS & 1) {
        const uint32_t st = __reduce_add_sync(0xffffffffu, cnt.steps);
        const uint32_t te = __reduce_add_sync(0xffffffffu, cnt.tests);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(counters + 1, (unsigned long long)st);
            atomicAdd(counters + 2, (unsigned long long)te);
        }
    }
}

// The k-th pixel of a w x h image in warp-tile order: when the sides are
// multiples of 16 and 8, each run of 128 takes a 16 x 8 region and each run
// of 32 an 8 x 4 tile of it, so a warp's camera rays (and the paths they
// start) stay close together; otherwise pixel k. Which thread traces a
// pixel does not change what is traced there. tile_px: thread k's pixel
// offset in a launch, tiled only over a whole frame.
__device__ __forceinline__ uint32_t tile_order(uint32_t w, uint32_t h, uint32_t k) {
    if ((w & 15u) != 0u || (h & 7u) != 0u) return k;
    const uint32_t block = k >> 7, warp = (k >> 5) & 3u, lane = k & 31u;
    const uint32_t bx = block % (w >> 4), by = block / (w >> 4);
    const uint32_t x = bx * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t y = by * 8u + (warp >> 1) * 4u + (lane >> 3);
    return y * w + x;
}
__device__ __forceinline__ uint32_t tile_px(const Frame& F, uint32_t k, uint32_t first, uint32_t count) {
    if (first != 0u || count != F.w * F.h) return k;
    return tile_order(F.w, F.h, k);
}

// MINB: resident 128-thread blocks per SM the register budget is set for
// (4: 128 registers a thread; 3: 168; 2: 255 — fewer warps, fewer spills;
// 5: 96, 6: 80, 8: 64, 10: 48, 12: 40, 16: 32 — more warps to hide the
// walk's loads, more spills).
template <int STATS, int MINB = 4, bool SYNC = false>
__global__ void __launch_bounds__(128, MINB) k_render(Scene S, Frame F, f3 sun, uint32_t* __restrict__ px,
                                                  uint32_t first, uint32_t count, unsigned long long* counters) {
    setup(S, F);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    Count cnt{0, 0, 0};
    if (F.adapt_list) {
        // shade.wgsl:44-50: thread k takes the k-th pixel still open
        if (k < px[34u * F.n]) render_px<STATS, SYNC>(S, F, sun, px, px[32u * F.n + k], cnt);
    } else if (k < count) {
        render_px<STATS, SYNC>(S, F, sun, px, first + tile_px(F, k, first, count), cnt);
    }
    flush_counts<STATS>(cnt, counters);
}

// show.wgsl: the display step of emit on its own, over the linear sums
// already in the image (Tracer::show writes a composited image there):
// the view transform of the mean over the samples that met something,
// the overlay laid over by its coverage, the packed pixel.
__global__ void k_show(uint32_t* __restrict__ px, uint32_t n, float exposure, float gamma) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float k = (float)max(px[31u * n + i], 1u);
    f3 l, gs;
    ld3(px, 1 * n, i, l);
    ld3(px, 20 * n, i, gs);
    const float cov = __uint_as_float(px[23u * n + i]);
    const float film = __uint_as_float(px[24u * n + i]);
    const float gone = __uint_as_float(px[33u * n + i]);
    const f3 shown = view_transform_std(l / fmaxf(k - gone, 1.0f), exposure, gamma) * (1.0f - cov / k) + gs / k;
    st3(px, 4 * n, i, shown);
    px[i] = pack_rgba(shown, film / k);
}

// ---- Adaptive Sampling (adapt.wgsl, gather.wgsl) ----

// adapt.wgsl's main: Cycles' convergence check at the end of `sample`, a
// step boundary past the minimum. The full and half images estimate the
// same mean; their disagreement scaled by the pixel's own sample count and
// normalised by its intensity (by its square root below 1) is the error.
__global__ void k_adapt_check(uint32_t* __restrict__ px, uint32_t n, float thr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || px[29u * n + i] != 0u) return;
    const uint32_t a = n + 3u * i, x = 26u * n + 3u * i;
    const f3 full = mk(__uint_as_float(px[a]), __uint_as_float(px[a + 1u]), __uint_as_float(px[a + 2u]));
    const f3 half = mk(__uint_as_float(px[x]), __uint_as_float(px[x + 1u]), __uint_as_float(px[x + 2u]));
    const uint32_t taken = max(px[31u * n + i], 1u);
    const float scale = 1.0f / (float)taken;
    const f3 d = mk(fabsf(full.x - half.x), fabsf(full.y - half.y), fabsf(full.z - half.z));
    const float error_difference = (d.x + d.y + d.z) * scale;
    const float intensity = (full.x + full.y + full.z) * scale;
    const float error_normalize = intensity < 1.0f ? sqrtf(intensity) : intensity;
    const float error = error_difference / (0.0001f + error_normalize);
    if (error < thr) px[29u * n + i] = 1u;
}

// adapt.wgsl's dilate: a pixel counts as settled only when it and its four
// neighbours are; the flag the tracer obeys.
__global__ void k_adapt_dilate(uint32_t* __restrict__ px, uint32_t w, uint32_t h) {
    const uint32_t n = w * h, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t x = i % w, y = i / w;
    const uint32_t* f = px + 29u * n;
    uint32_t all = f[i];
    if (x > 0u) all = min(all, f[i - 1u]);
    if (x + 1u < w) all = min(all, f[i + 1u]);
    if (y > 0u) all = min(all, f[i - w]);
    if (y + 1u < h) all = min(all, f[i + w]);
    px[30u * n + i] = all;
}

// gather.wgsl: the list of pixels not settled, each block appending its
// open pixels as one run in the order it visits them — the warp tiles'
// order (tile_order), so a warp of the list launch traces neighbouring
// pixels while most are open. The list's order decides only which thread
// traces which pixel, never a result.
__global__ void __launch_bounds__(256) k_adapt_gather(uint32_t* __restrict__ px, uint32_t w, uint32_t h) {
    __shared__ uint32_t held, run;
    if (threadIdx.x == 0) held = 0u;
    __syncthreads();
    const uint32_t n = w * h;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = k < n ? tile_order(w, h, k) : k;
    const bool open = k < n && px[30u * n + i] == 0u;
    const unsigned ballot = __ballot_sync(0xffffffffu, open);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0 && ballot) base = atomicAdd(&held, (uint32_t)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    __syncthreads();
    if (threadIdx.x == 0) run = atomicAdd(px + 34u * n, held);
    __syncthreads();
    if (open) px[32u * n + run + base + __popc(ballot & ((1u << lane) - 1u))] = i;
}

// ---- many scenes in one persistent launch ----
//
// A job is one tracer's frame: its scene, camera frame, image and ray
// counters. Its pixels are cut into tiles of 32 (one warp each); the tiles
// of all jobs are numbered in one range, the costliest jobs first. Each
// warp of a grid sized to the resident capacity takes the next tile from a
// counter, finds its job by binary search over the jobs' first tiles, copies
// the job record to its slot of shared memory, and renders the tile's
// pixels: the same per-pixel computation as k_render, so every job's image
// is bit for bit its single-scene render.
struct Job {
    Scene S;
    Frame F;
    f3 sun;
    uint32_t* px;
    unsigned long long* counters;
    uint32_t tile0;  // first tile of this job in the launch's numbering
    uint32_t npx;
};

// Lane `lane` of a job's warp tile q: an 8 x 4 block of pixels when the
// image's sides are multiples of 8 and 4 (q counts the blocks row by row),
// else the 32 pixels from q * 32 on.
__device__ __forceinline__ uint32_t warp_tile_px(const Frame& F, uint32_t q, uint32_t lane) {
    if ((F.w & 7u) != 0u || (F.h & 3u) != 0u) return q * 32u + lane;
    const uint32_t across = F.w >> 3;
    return ((q / across) * 4u + (lane >> 3)) * F.w + (q % across) * 8u + (lane & 7u);
}

// Registers are budgeted for RES resident threads an SM: 1536 (40 a
// thread) or every thread slot, 2048 (32 a thread). The walk is
// latency-bound, so more resident warps pay although they spill more.
template <int STATS, int THREADS, int RES>
__global__ void __launch_bounds__(THREADS, RES / THREADS) k_render_batch(const Job* __restrict__ jobs, uint32_t njobs,
                                                                        uint32_t ntiles, uint32_t* next) {
    constexpr int WARPS = THREADS / 32;
    constexpr int WORDS = (int)(sizeof(Job) / 4);
    __shared__ __align__(16) Job sj[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Job& J = sj[warp];
    uint32_t cur = 0xFFFFFFFFu;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(next, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ntiles) break;
        uint32_t lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&jobs[mid].tile0) <= t) lo = mid;
            else hi = mid - 1;
        }
        if (lo != cur) {
            __syncwarp();
            const uint32_t* src = (const uint32_t*)(jobs + lo);
            uint32_t* dst = (uint32_t*)&J;
            for (int k = lane; k < WORDS; k += 32) dst[k] = __ldg(src + k);
            __syncwarp();
            if (lane == 0) setup(J.S, J.F);
            __syncwarp();
            cur = lo;
        }
        const uint32_t p = warp_tile_px(J.F, t - J.tile0, (uint32_t)lane);
        Count cnt{0, 0, 0};
        if (p < J.npx) render_px<STATS>(J.S, J.F, J.sun, J.px, p, cnt);
        flush_counts<STATS>(cnt, J.counters);
    }
}

// ---- the persistent state-machine render (one trace site) ----
//
// The same computation as k_render, restructured so every lane reaches the
// traversal at one program point: a lane's work between two traces is a
// phase of a state machine, and the loop head traces whatever ray the
// lane's phase left (closest hit or shadow). Lanes whose paths are at
// different points of the bounce loop then still walk the tree together.
// direct()'s shadow rays are traced after all its light queries: the queries
// draw every random number first and the shadow results only enter the sum,
// so the draws and the sum happen in the reference's order. Lanes fetch
// pixels from a counter and take each pixel's samples in order, so per-pixel
// sums are added in frame order, as the reference's per-sample loop adds them.

enum Phase : uint32_t {
    PH_TRACE = 0,  // a ray is set: trace it, then go to `after`
    PH_DONE,
    PH_BEGIN_SAMPLE,
    PH_ON_BOUNCE,
    PH_SHINE_OR_LOBE,
    PH_LOBE,
    PH_IND_STEP,
    PH_ON_IND_HIT,
    PH_IND_AFTER_DIRECT,
    PH_ON_IND_AO,
    PH_AFTER_INDIRECT,
    PH_GLOSSY,
    PH_ON_GLOSSY,
    PH_AFTER_GLOSSY,
    PH_END_SHADING,
    PH_EMIT_END,
    PH_FINISH_SAMPLE,
    PH_DIRECT_NEXT,
    PH_ON_SHADOW,
    PH_AFTER_DIRECT,
};

enum Cont : uint32_t { C_OPAQUE = 0, C_SHINE = 1, C_IND = 2, C_BOUNCE_LIGHT = 3 };

struct Path {
    // the ray the loop head traces next, and the phase that takes its hit
    f3 ro, rd;
    float rtmax;
    uint32_t rany, after;
    // pixel and sample
    uint32_t i, frame, frame_end, seed;
    f3 o, d, col, thr;
    uint32_t bounce, n_see, n_through;
    // the camera-path hit being shaded
    f3 hit, past, base, ng;
    uint32_t front;
    float trans, metal, ior, opaque, p_diffuse;
    uint32_t take_diffuse;
    Surf s;
    f3 c, bounced, diffuse_weight, aval;
    // glossy ray
    f3 fres;
    float ggx_a, cos_no;
    // direct(): queries with light, traced in order (four named slots, so no
    // array is indexed at run time and the state can stay in registers)
    f3 dpos, dsum;
    f3 qc0, qc1, qc2, qc3, qd0, qd1, qd2, qd3;
    float ql0, ql1, ql2, ql3;
    uint32_t qn, qk, cont;

    __device__ __forceinline__ void put(uint32_t k, f3 c, f3 d, float l) {
        if (k == 0) { qc0 = c; qd0 = d; ql0 = l; }
        else if (k == 1) { qc1 = c; qd1 = d; ql1 = l; }
        else if (k == 2) { qc2 = c; qd2 = d; ql2 = l; }
        else { qc3 = c; qd3 = d; ql3 = l; }
    }
    __device__ __forceinline__ f3 qc(uint32_t k) const { return k == 0 ? qc0 : (k == 1 ? qc1 : (k == 2 ? qc2 : qc3)); }
    __device__ __forceinline__ f3 qd(uint32_t k) const { return k == 0 ? qd0 : (k == 1 ? qd1 : (k == 2 ? qd2 : qd3)); }
    __device__ __forceinline__ float ql(uint32_t k) const { return k == 0 ? ql0 : (k == 1 ? ql1 : (k == 2 ? ql2 : ql3)); }
    // indirect()
    f3 iacc, ithr, iorg, inrm, idir, ibase, ialbedo, ihit, ing;
    uint32_t ib, idepth, ithrough, ibounce;
    float imin_pdf, ipb, inear, itw, iht;
    // bounce_light()
    f3 balbedo, bemit;
};

__device__ __forceinline__ uint32_t set_ray(Path& P, f3 o, f3 d, float tmax, bool any, uint32_t after) {
    P.ro = o;
    P.rd = d;
    P.rtmax = tmax;
    P.rany = any ? 1u : 0u;
    P.after = after;
    return PH_TRACE;
}

// direct() up to its shadow rays: every query (and its draws) in order.
template <int STATS>
__device__ __forceinline__ uint32_t start_direct(const Scene& S, const Frame& F, Path& P, const Surf& s, uint32_t cont,
                                                 f3 sun) {
    const bool rig = uses_rig(F);
    P.dsum = rig ? rig_fill(F, s) : mk(0.0f);
    P.qn = 0;
    for (uint32_t k = 0; k < 4u; k++) {
        Shadowed q = unshadowed();
        if (k == 0u) {
            q = rig ? rig_query(F, 0u, s, P.seed, sun) : lamp_query(F, s, P.seed);
        } else if (k == 1u) {
            if (rig) q = rig_query(F, 1u, s, P.seed, sun);
        } else if (k == 2u) {
            q = glow_query<STATS>(S, s, P.seed);
        }
        if (maxc(q.c) > 0.0f) {
            P.put(P.qn, q.c, q.dir, q.dist);
            P.qn++;
        }
    }
    P.dpos = s.pos;
    P.qk = 0;
    P.cont = cont;
    return PH_DIRECT_NEXT;
}

template <int STATS>
__device__ __forceinline__ uint32_t step(const Scene& S, const Frame& F, Path& P, uint32_t ph, const Hit& h, f3 sun,
                                         Sums& acc) {
    const uint32_t see_through = 8u, through = 8u;
    const uint32_t passes = see_through + through + 1u;
    switch (ph) {
        case PH_BEGIN_SAMPLE: {
            P.seed = hash(P.i * 9781u + P.frame * 6271u + 1u);
            const CamRay cr = camera_ray(F, P.i, P.seed);
            P.o = cr.o;
            P.d = cr.d;
            acc.outline = 0;
            P.col = mk(0.0f);
            P.thr = mk(1.0f);
            P.bounce = P.n_see = P.n_through = 0;
            return set_ray(P, P.o, P.d, INF, false, PH_ON_BOUNCE);
        }
        case PH_ON_BOUNCE: {
            if (h.tri == NONE) {
                if (P.bounce == 0u) {
                    const float across = (float)(P.i % F.w) / fmaxf((float)F.w * 0.5f, 1.0f);
                    const float lift = F.sky[3] * (1.0f - clampf(across, 0.0f, 1.0f));
                    const f3 sky = mk(F.sky[0] + lift, F.sky[1] + lift, F.sky[2] + lift);
                    acc.alb += mk(srgb_to_linear1(sky.x), srgb_to_linear1(sky.y), srgb_to_linear1(sky.z));
                    acc.nrm += -P.d;
                    acc.dep += -1.0f;
                    acc.gone += 1.0f;
                    acc.count += 1u;
                    acc.film += 1.0f;
                    acc.lin += mk(0.0f);
                    if ((STATS & MODE_FULL) && F.grid > 0.0f) {
                        const Over gr = grid_over(F, P.o, P.d, INF);
                        acc.grid += sky * (1.0f - gr.a) + gr.c;
                    } else {
                        acc.grid += sky * (1.0f - 0.0f) + mk(0.0f);
                    }
                    acc.cov += 1.0f;
                    return PH_FINISH_SAMPLE;
                }
                P.col += P.thr * env_at(F);
                return PH_EMIT_END;
            }
            if (P.bounce == 0u) {
                acc.outline = ((STATS & MODE_FULL) ? h.inst : 0u) + 1u;
                if ((STATS & MODE_FULL) && F.grid > 0.0f) {  // emit's overlay, as in sample()
                    const Over gr = grid_over(F, P.o, P.d, h.t);
                    acc.grid += gr.c;
                    acc.cov += gr.a;
                }
            }
            const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
            const Mat t = mat_at(S, g.mat);
            const float w = 1.0f - h.u - h.v;
            const f3 hit = P.o + P.d * h.t;
            const f3 ngw = normalize(cross(g.b - g.a, g.c - g.a));
            const f3 ng0 = g.mirror ? -ngw : ngw;  // world_ng
            const bool front = dot(ng0, P.d) < 0.0f;
            const f3 ng = front ? ng0 : -ng0;
            f3 n = g.na * w + g.nb * h.u + g.nc * h.v;
            n = dot(n, n) > 1e-12f ? normalize(n) * (front ? 1.0f : -1.0f) : ng;
            if (dot(n, -P.d) < 0.0f) n = ng;
            const f3 off = ng * hit_lift(F, h.t);
            const f3 past = ng * through_lift(F, hit, h.t);
            const f3 pos = hit + off;
            const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
            if (P.bounce == 0u) {
                acc.alb += base;
                acc.nrm += n;
                acc.dep += h.t;
            }
            if (rnd(P.seed) >= t.color.w) {
                P.n_see++;
                if (P.n_see > see_through) return PH_EMIT_END;
                P.o = hit - past;
                P.bounce++;
                if (P.bounce < passes) return set_ray(P, P.o, P.d, INF, false, PH_ON_BOUNCE);
                return PH_EMIT_END;
            }
            P.col += P.thr * t.emit;
            const float bleed = scatter_bleed(t.sss, t.sss_radius);
            const f3 fd = dielectric_f0(t.ior);
            f3 diffuse = base * (1.0f - t.metal);
            if (maxc(diffuse) > 0.0f)
                diffuse *= under_layer_real(t.ior, fmaxf(t.rough, 0.04f), fmaxf(dot(n, -P.d), 1e-4f));
            P.s = Surf{pos,   n,      -P.d,   diffuse,    vmix(fd, base, t.metal), fmaxf(t.rough, 0.04f),
                       bleed, scatter_tint(t.sss_radius), t.sheen, t.sheen_rough, t.sheen_tint,
                       t.coat, t.coat_rough, t.ior, 1.0f - t.metal};
            P.hit = hit;
            P.past = past;
            P.base = base;
            P.ng = ng;
            P.front = front ? 1u : 0u;
            P.trans = t.trans;
            P.metal = t.metal;
            P.ior = t.ior;
            P.opaque = 1.0f - t.trans * (1.0f - t.metal);
            P.c = mk(0.0f);
            if (P.opaque > 0.0f) return start_direct<STATS>(S, F, P, P.s, C_OPAQUE, sun);
            return PH_SHINE_OR_LOBE;
        }
        case PH_SHINE_OR_LOBE: {
            if (P.opaque < 1.0f) {
                const Surf shine{P.s.pos, P.s.n, P.s.v, mk(0.0f), P.s.f0, P.s.rough, 0.0f, mk(1.0f), 0.0f,
                                 P.s.sheen_rough, P.s.sheen_tint, P.s.coat, P.s.coat_rough, P.s.eta, P.s.dielectric};
                return start_direct<STATS>(S, F, P, shine, C_SHINE, sun);
            }
            return PH_LOBE;
        }
        case PH_LOBE: {
            P.c = clamp_light(P.c, F.limit_d);
            P.bounced = mk(0.0f);
            const Surf& s = P.s;
            const float bleed = s.bleed;
            P.diffuse_weight = vmix(s.albedo, s.albedo * s.sss_tint, bleed) * P.opaque;
            const f3 lw = mk(0.2126f, 0.7152f, 0.0722f);
            const float ndv = fmaxf(dot(s.n, -P.d), 1e-4f);
            const f3 gloss_guess = s.f0 + (mk(1.0f) - s.f0) * pm_pow(1.0f - ndv, 5.0f);
            const float pd = dot(vmax(P.diffuse_weight, mk(0.0f)), lw);
            const float pg = dot(gloss_guess, lw);
            float p_diffuse = pd + pg > 0.0f ? pd / (pd + pg) : 1.0f;
            if (pd > 0.0f && pg > 0.0f) p_diffuse = clampf(p_diffuse, 0.15f, 0.85f);
            P.p_diffuse = p_diffuse;
            P.take_diffuse = rnd(P.seed) < p_diffuse ? 1u : 0u;
            if (!(P.take_diffuse && pd > 0.0f)) return PH_GLOSSY;
            // indirect(pos, n, seed, diffuse_on)
            const bool lit = dot(F.env, F.env) > 0.0f;
            if (S.lamp_count == 0u && !lit) {
                const f3 dir = cosine_dir(s.n, P.seed);
                if (F.env.x == 0.0f && F.env.y == 0.0f && F.env.z == 0.0f) {
                    P.aval = mk(0.0f);
                    return PH_AFTER_INDIRECT;
                }
                return set_ray(P, s.pos, dir, F.ao, true, PH_ON_IND_AO);
            }
            P.idepth = F.bounces != 0u ? F.bounces : 1u;
            P.ibounce = 1u;
            P.iacc = mk(0.0f);
            P.ithr = mk(1.0f);
            P.iorg = s.pos;
            P.inrm = s.n;
            P.imin_pdf = 3.0e38f;
            P.ithrough = 0u;
            P.idir = mk(0.0f, 0.0f, 1.0f);
            P.ipb = 1.0f;
            P.ib = 0;
            return PH_IND_STEP;
        }
        case PH_IND_STEP: {
            if (P.ib >= P.idepth) {
                P.aval = P.iacc;
                return PH_AFTER_INDIRECT;
            }
            if (!P.ithrough) {
                P.idir = cosine_dir(P.inrm, P.seed);
                P.ipb = fmaxf(dot(P.inrm, P.idir), 0.0f) / PI;
            }
            P.ithrough = 0u;
            P.imin_pdf = fminf(P.imin_pdf, P.ipb);
            return set_ray(P, P.iorg, P.idir, INF, false, PH_ON_IND_HIT);
        }
        case PH_ON_IND_HIT: {
            if (h.tri == NONE) {
                P.iacc += P.ithr * env_at(F) * 1.0f;
                P.aval = P.iacc;
                return PH_AFTER_INDIRECT;
            }
            if (!P.ibounce) {
                P.aval = P.iacc;
                return PH_AFTER_INDIRECT;
            }
            const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
            const Mat t = mat_at(S, g.mat);
            const f3 dir = P.idir;
            const f3 ng0 = normalize(cross(g.b - g.a, g.c - g.a));
            const f3 ng = dot(ng0, dir) < 0.0f ? ng0 : -ng0;
            const f3 hit = P.iorg + dir * h.t + ng * (F.eps + h.t * 1e-5f);
            const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
            const float rough = fmaxf(t.rough, glossy_floor());
            const f3 fd = dielectric_f0(t.ior);
            const float tw = t.trans * (1.0f - t.metal);
            f3 albedo = base * (1.0f - t.metal) * (1.0f - tw);
            if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxf(dot(ng, -dir), 1e-4f));
            P.iacc += P.ithr * glow_mis<STATS>(S, g, t.emit, h, P.inrm, dir);
            const bool lit = dot(F.env, F.env) > 0.0f;
            P.inear = (!lit && h.t <= F.ao) ? 0.25f : 1.0f;
            P.itw = tw;
            P.ibase = base;
            P.ialbedo = albedo;
            P.ihit = hit;
            P.ing = ng;
            P.iht = h.t;
            const Surf si = plain_surf(hit, ng, -dir, albedo, vmix(fd, base, t.metal), rough);
            return start_direct<STATS>(S, F, P, si, C_IND, sun);
        }
        case PH_IND_AFTER_DIRECT: {
            if (P.itw > 0.0f && rnd(P.seed) < P.itw) {
                P.ithr *= mk(sqrtf(P.ibase.x), sqrtf(P.ibase.y), sqrtf(P.ibase.z));
                const f3 at = P.iorg + P.idir * P.iht;
                P.iorg = at - P.ing * through_lift(F, at, P.iht);
                P.ithrough = 1u;
                P.ib++;
                return PH_IND_STEP;
            }
            P.ithr *= P.ialbedo;
            if (P.ib + 1u < P.idepth) {
                const float keep = clampf(maxc(P.ithr), 0.0f, 0.95f);
                if (keep < 1e-4f || rnd(P.seed) > keep) {
                    P.aval = P.iacc;
                    return PH_AFTER_INDIRECT;
                }
                P.ithr = P.ithr / keep;
            }
            P.iorg = P.ihit;
            P.inrm = P.ing;
            P.ib++;
            return PH_IND_STEP;
        }
        case PH_ON_IND_AO: {
            const float vis = h.tri != NONE ? 0.0f : 1.0f;
            P.aval = env_at(F) * mixf(0.25f, 1.0f, vis);
            return PH_AFTER_INDIRECT;
        }
        case PH_AFTER_INDIRECT: {
            P.bounced += P.diffuse_weight * P.aval / P.p_diffuse;
            return PH_GLOSSY;
        }
        case PH_GLOSSY: {
            const Surf& s = P.s;
            const f3 v = -P.d;
            const f3 tx = normalize(onb(s.n, 1.0f, 0.0f));
            const f3 ty = cross(s.n, tx);
            P.ggx_a = s.rough * s.rough;
            const f3 wi_local = mk(dot(v, tx), dot(v, ty), dot(v, s.n));
            const float r1 = rnd(P.seed);
            const float r2 = rnd(P.seed);
            const f3 h_local = ggx_sample_vndf(wi_local, P.ggx_a, r1, r2);
            const f3 hw = normalize(tx * h_local.x + ty * h_local.y + s.n * h_local.z);
            const f3 refl = reflect(P.d, hw);
            const float cos_hi = fmaxf(dot(hw, v), 0.0f);
            P.cos_no = dot(s.n, refl);
            P.fres = fresnel_of(s, cos_hi);
            if (!P.take_diffuse && dot(refl, P.ng) > 0.0f && cos_hi > 0.0f && P.cos_no > 0.0f)
                return set_ray(P, s.pos, refl, INF, false, PH_ON_GLOSSY);
            return PH_END_SHADING;
        }
        case PH_ON_GLOSSY: {
            if (h.tri == NONE) {
                P.aval = env_at(F);
                return PH_AFTER_GLOSSY;
            }
            // bounce_light (integrate.wgsl:236-250) up to its direct().
            const Geo g = geo_at<STATS>(S, h.tri, (STATS & MODE_FULL) ? h.inst : 0u);
            const Mat t = mat_at(S, g.mat);
            const f3 d = P.rd;
            const f3 ng0 = normalize(cross(g.b - g.a, g.c - g.a));
            const f3 ng = dot(ng0, d) < 0.0f ? ng0 : -ng0;
            const f3 pos = P.ro + d * h.t + ng * (F.eps + h.t * 1e-5f);
            const f3 base = vmax(mk(t.color.x, t.color.y, t.color.z), mk(0.0f));
            const float rough = fmaxf(t.rough, glossy_floor());
            const f3 fd = dielectric_f0(t.ior);
            f3 albedo = base * (1.0f - t.metal);
            if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxf(dot(ng, -d), 1e-4f));
            const Surf s2 = plain_surf(pos, ng, -d, albedo, vmix(fd, base, t.metal), rough);
            P.balbedo = s2.albedo;
            P.bemit = t.emit;
            return start_direct<STATS>(S, F, P, s2, C_BOUNCE_LIGHT, sun);
        }
        case PH_AFTER_GLOSSY: {
            const Surf& s = P.s;
            P.bounced += P.fres * P.aval * ggx_weight(P.ggx_a * P.ggx_a, fmaxf(dot(s.n, -P.d), 1e-4f), P.cos_no) *
                         1.0f / (1.0f - P.p_diffuse);
            return PH_END_SHADING;
        }
        case PH_END_SHADING: {
            P.c += clamp_light(P.bounced, F.limit_i);
            P.col += P.thr * P.c;
            const float tw = P.trans * (1.0f - P.metal);
            if (tw <= 0.0f) return PH_EMIT_END;
            P.n_through++;
            if (P.n_through > through) return PH_EMIT_END;
            const float eta = P.front ? 1.0f / P.ior : P.ior;
            f3 nd = refract(P.d, P.s.n, eta);
            if (dot(nd, nd) < 1e-6f) {
                nd = reflect(P.d, P.s.n);
                P.o = P.hit + P.past;
                P.thr *= tw;
            } else {
                P.o = P.hit - P.past;
                P.thr *= mk(sqrtf(P.base.x), sqrtf(P.base.y), sqrtf(P.base.z)) * tw * (mk(1.0f) - P.fres);
            }
            P.d = cone_dir(normalize(nd), P.s.rough * P.s.rough, P.seed);
            if (maxc(P.thr) < 0.01f) return PH_EMIT_END;
            P.bounce++;
            if (P.bounce < passes) return set_ray(P, P.o, P.d, INF, false, PH_ON_BOUNCE);
            return PH_EMIT_END;
        }
        case PH_EMIT_END: {
            acc.gone += 0.0f;
            acc.count += 1u;
            acc.film += 1.0f;
            acc.lin += P.col;
            return PH_FINISH_SAMPLE;
        }
        case PH_DIRECT_NEXT: {
            if (P.qk < P.qn) return set_ray(P, P.dpos, P.qd(P.qk), P.ql(P.qk), true, PH_ON_SHADOW);
            return PH_AFTER_DIRECT;
        }
        case PH_ON_SHADOW: {
            const float vis = h.tri != NONE ? 0.0f : 1.0f;
            P.dsum += P.qc(P.qk) * vis;
            P.qk++;
            return PH_DIRECT_NEXT;
        }
        case PH_AFTER_DIRECT: {
            const f3 D = P.dsum;
            if (P.cont == C_OPAQUE) {
                P.c = D * P.opaque;
                return PH_SHINE_OR_LOBE;
            }
            if (P.cont == C_SHINE) {
                P.c += D * (1.0f - P.opaque);
                return PH_LOBE;
            }
            if (P.cont == C_IND) {
                P.iacc += P.ithr * D * P.inear;
                return PH_IND_AFTER_DIRECT;
            }
            P.aval = D + P.balbedo * env_at(F) * 0.8f + P.bemit;
            return PH_AFTER_GLOSSY;
        }
    }
    return PH_DONE;
}

__device__ __forceinline__ void load_sums(const uint32_t* px, uint32_t n, uint32_t i, bool keep, Sums& acc) {
    if (keep) {
        ld3(px, 1 * n, i, acc.lin);
        ld3(px, 20 * n, i, acc.grid);
        ld3(px, 7 * n, i, acc.alb);
        ld3(px, 10 * n, i, acc.nrm);
        acc.cov = __uint_as_float(px[23 * n + i]);
        acc.film = __uint_as_float(px[24 * n + i]);
        acc.gone = __uint_as_float(px[33 * n + i]);
        acc.dep = __uint_as_float(px[13 * n + i]);
        acc.count = px[31 * n + i];
    } else {
        acc.lin = acc.grid = acc.alb = acc.nrm = mk(0.0f);
        acc.cov = acc.film = acc.gone = acc.dep = 0.0f;
        acc.count = 0;
    }
    acc.outline = 0;
}

__device__ __forceinline__ void store_sums(uint32_t* px, uint32_t n, uint32_t i, bool first_frame, const Sums& acc,
                                           const Frame& F) {
    if (first_frame) {
        px[29 * n + i] = 0u;
        px[30 * n + i] = 0u;
    }
    st3(px, 1 * n, i, acc.lin);
    st3(px, 20 * n, i, acc.grid);
    st3(px, 7 * n, i, acc.alb);
    st3(px, 10 * n, i, acc.nrm);
    px[23 * n + i] = __float_as_uint(acc.cov);
    px[24 * n + i] = __float_as_uint(acc.film);
    px[33 * n + i] = __float_as_uint(acc.gone);
    px[13 * n + i] = __float_as_uint(acc.dep);
    px[31 * n + i] = acc.count;
    px[25 * n + i] = acc.outline;
    const float kk = (float)acc.count;
    const f3 shown = view_transform_std(acc.lin / fmaxf(kk - acc.gone, 1.0f), F.exposure, F.gamma) *
                         (1.0f - acc.cov / kk) +
                     acc.grid / kk;
    st3(px, 4 * n, i, shown);
    px[i] = pack_rgba(shown, acc.film / kk);
}

// Persistent: every lane takes pixels from `next` until [first, first +
// count) is done, tracing all of a pixel's samples in frame order.
template <int STATS, int MINB>
__global__ void __launch_bounds__(128, MINB) k_render_sm(Scene S, Frame F, f3 sun, uint32_t* __restrict__ px, uint32_t first,
                                                  uint32_t count, uint32_t* next, unsigned long long* counters) {
    setup(S, F);
    Count cnt{0, 0, 0};
    Path P;
    Sums acc;
    uint32_t ph = PH_DONE;
    uint32_t k = atomicAdd(next, 1u);
    if (k < count) {
        P.i = first + k;
        P.frame = F.frame0;
        P.frame_end = F.frame0 + F.spp;
        load_sums(px, F.n, P.i, F.frame0 > 0u, acc);
        ph = F.spp > 0u ? (uint32_t)PH_BEGIN_SAMPLE : (uint32_t)PH_FINISH_SAMPLE;
    }
    Hit h{INF, NONE, 0.0f, 0.0f, 0u};
    for (;;) {
        // run phases until the lane needs a ray or runs out of pixels
        while (ph != PH_TRACE && ph != PH_DONE) {
            if (ph == PH_FINISH_SAMPLE) {
                P.frame++;
                if (P.frame < P.frame_end) {
                    ph = PH_BEGIN_SAMPLE;
                    continue;
                }
                store_sums(px, F.n, P.i, F.frame0 == 0u, acc, F);
                k = atomicAdd(next, 1u);
                if (k >= count) {
                    ph = PH_DONE;
                    break;
                }
                P.i = first + k;
                P.frame = F.frame0;
                load_sums(px, F.n, P.i, F.frame0 > 0u, acc);
                ph = PH_BEGIN_SAMPLE;
                continue;
            }
            ph = step<STATS>(S, F, P, ph, h, sun, acc);
        }
        if (__all_sync(0xffffffffu, ph == PH_DONE)) break;
        if (ph == PH_TRACE) {
            h = walk_mode<STATS>(S, P.ro, P.rd, P.rtmax, P.rany != 0u, cnt);
            ph = P.after;
        }
    }
    const uint32_t tot = __reduce_add_sync(0xffffffffu, cnt.rays);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(counters, (unsigned long long)tot);
    if (STATS & 1) {
        const uint32_t st = __reduce_add_sync(0xffffffffu, cnt.steps);
        const uint32_t te = __reduce_add_sync(0xffffffffu, cnt.tests);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(counters + 1, (unsigned long long)st);
            atomicAdd(counters + 2, (unsigned long long)te);
        }
    }
}

// ---- the wavefront render: path state in memory, rays queued by type ----
//
// The state machine above with its one trace site cut out of the kernel:
// a logic kernel runs every path slot's phases (step(), the same code) until
// the path needs a ray, then appends the slot to the queue of its ray's
// type — primary (a sample's camera ray), extension (any other closest-hit
// ray) or shadow (any hit) — with one atomic a warp (ballot compaction), and
// stores the slot's state; separate walk kernels then trace each queue alone,
// closest-hit or any-hit, at full occupancy with no shading state, and write
// each slot's hit; the next logic pass resumes every slot at its ray's
// phase. A slot takes pixels from a counter and a pixel's samples in frame
// order, so each pixel's sums are added in the reference's order: the image
// is the megakernel's bit for bit.

struct WfSlot {
    Path P;
    Sums acc;
    uint32_t ph;  // the phase to resume at (its ray's hit is in the hit buffer)
};
constexpr uint32_t WF_WORDS = (uint32_t)((sizeof(WfSlot) + 3) / 4);
constexpr uint32_t WF_START = 0xFFFFFFF0u;  // a slot that has yet to take its first pixel
enum : uint32_t { Q_PRIMARY = 0, Q_EXTEND = 1, Q_SHADOW = 2 };

// The slot's state, one 32-bit word of every slot after another (word k of
// slot s at words[k * nslots + s]: a warp's loads of a word coalesce).
__device__ __forceinline__ void wf_load(const uint32_t* __restrict__ words, uint32_t nslots, uint32_t s, WfSlot& w) {
    uint32_t* d = reinterpret_cast<uint32_t*>(&w);
#pragma unroll 8
    for (uint32_t k = 0; k < WF_WORDS; k++) d[k] = words[(size_t)k * nslots + s];
}

__device__ __forceinline__ void wf_store(uint32_t* __restrict__ words, uint32_t nslots, uint32_t s, const WfSlot& w) {
    const uint32_t* d = reinterpret_cast<const uint32_t*>(&w);
#pragma unroll 8
    for (uint32_t k = 0; k < WF_WORDS; k++) words[(size_t)k * nslots + s] = d[k];
}

__global__ void k_wf_init(uint32_t* __restrict__ words, uint32_t nslots) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslots) words[(size_t)(offsetof(WfSlot, ph) / 4) * nslots + s] = WF_START;
}

// Appends slot s to queue q with one atomic per warp and queue (the lanes
// of a warp that push to the same queue share it).
__device__ __forceinline__ void wf_push(uint32_t q, bool push, uint32_t s, uint32_t* __restrict__ queues,
                                        uint32_t* __restrict__ lens, uint32_t nslots) {
    const unsigned all = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t t = 0; t < 3u; t++) {
        const unsigned m = __ballot_sync(all, push && q == t);
        if (!m) continue;
        const uint32_t leader = __ffs(m) - 1u;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(lens + t, (uint32_t)__popc(m));
        base = __shfl_sync(all, base, leader);
        if (push && q == t) queues[(size_t)t * nslots + base + __popc(m & ((1u << lane) - 1u))] = s;
    }
}

template <int STATS>
__global__ void __launch_bounds__(128) k_wf_logic(Scene S, Frame F, f3 sun, uint32_t* __restrict__ px, uint32_t first,
                                                  uint32_t count, uint32_t* next, uint32_t* __restrict__ words,
                                                  uint32_t nslots, const float4* __restrict__ hits,
                                                  const uint32_t* __restrict__ hit_inst, float4* __restrict__ rays,
                                                  uint32_t* __restrict__ queues, uint32_t* __restrict__ lens) {
    setup(S, F);
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool push = false;
    uint32_t q = 0;
    if (s < nslots) {
        WfSlot w;
        const uint32_t ph0 = words[(size_t)(offsetof(WfSlot, ph) / 4) * nslots + s];
        if (ph0 != PH_DONE) {
            Path& P = w.P;
            Sums& acc = w.acc;
            // the next pixel from the counter, or PH_DONE
            auto fetch = [&]() -> uint32_t {
                const uint32_t k = atomicAdd(next, 1u);
                if (k >= count) return PH_DONE;
                P.i = first + k;
                P.frame = F.frame0;
                P.frame_end = F.frame0 + F.spp;
                load_sums(px, F.n, P.i, F.frame0 > 0u, acc);
                return F.spp > 0u ? (uint32_t)PH_BEGIN_SAMPLE : (uint32_t)PH_FINISH_SAMPLE;
            };
            uint32_t ph;
            Hit h{INF, NONE, 0.0f, 0.0f, 0u};
            if (ph0 == WF_START) {
                ph = fetch();
            } else {
                wf_load(words, nslots, s, w);
                ph = ph0;
                const float4 hv = __ldg(hits + s);
                h = Hit{hv.x, __float_as_uint(hv.y), hv.z, hv.w, (STATS & MODE_FULL) ? __ldg(hit_inst + s) : 0u};
            }
            while (ph != PH_TRACE && ph != PH_DONE) {
                if (ph == PH_FINISH_SAMPLE) {
                    P.frame++;
                    if (P.frame < P.frame_end) {
                        ph = PH_BEGIN_SAMPLE;
                        continue;
                    }
                    store_sums(px, F.n, P.i, F.frame0 == 0u, acc, F);
                    ph = fetch();
                    continue;
                }
                ph = step<STATS>(S, F, P, ph, h, sun, acc);
            }
            if (ph == PH_TRACE) {
                push = true;
                q = P.rany ? Q_SHADOW : ((P.after == PH_ON_BOUNCE && P.bounce == 0u) ? Q_PRIMARY : Q_EXTEND);
                rays[2 * (size_t)s] = make_float4(P.ro.x, P.ro.y, P.ro.z, P.rtmax);
                rays[2 * (size_t)s + 1] = make_float4(P.rd.x, P.rd.y, P.rd.z, 0.0f);
                w.ph = P.after;
                wf_store(words, nslots, s, w);
            } else {
                words[(size_t)(offsetof(WfSlot, ph) / 4) * nslots + s] = PH_DONE;
            }
        }
    }
    wf_push(q, push, s, queues, lens, nslots);
}

// One queue's rays, closest hit (ANY false) or any hit, each slot's hit
// written at the slot. Also counts rays (and STATS: steps, tests).
template <bool ANY, int STATS>
__global__ void __launch_bounds__(128) k_wf_walk(Scene S, const uint32_t* __restrict__ queue,
                                                 const uint32_t* __restrict__ len, const float4* __restrict__ rays,
                                                 float4* __restrict__ hits, uint32_t* __restrict__ hit_inst,
                                                 unsigned long long* counters) {
    load_info(S);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    Count cnt{0, 0, 0};
    if (k < *len) {
        const uint32_t s = __ldg(queue + k);
        const float4 a = __ldg(rays + 2 * (size_t)s), b = __ldg(rays + 2 * (size_t)s + 1);
        const Hit h = walk_mode<STATS>(S, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, ANY, cnt);
        hits[s] = make_float4(h.t, __uint_as_float(h.tri), h.u, h.v);
        if (STATS & MODE_FULL) hit_inst[s] = h.inst;
    }
    flush_counts<STATS>(cnt, counters);
}


// The render kernels of one mode M (MODE_STATS, MODE_FULL bits) at the
// tracer's kernel id, over pixels [first_px, first_px + count_px).


template <int M, int MINB>
int32_t launch_sm(const RenderLaunch& L) {
    int per_sm = 0;
    PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_sm<M, MINB>, 128, 0));
    const uint32_t grid = (uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)L.sms;
    const uint32_t blocks = std::min<uint32_t>(grid, (L.count + 127) / 128);
    PHX_CUDA(cudaMemsetAsync(L.next, 0, 4, L.s));
    k_render_sm<M, MINB><<<blocks, 128, 0, L.s>>>(L.S, L.F, L.sun, L.px, L.first, L.count, L.next, L.counters);
    return cuda_check(cudaGetLastError(), "render");
}

template <int M, int MINB, bool SYNC>
int32_t launch_mk(const RenderLaunch& L) {
    k_render<M, MINB, SYNC><<<(L.count + 127) / 128, 128, 0, L.s>>>(L.S, L.F, L.sun, L.px, L.first, L.count,
                                                                     L.counters);
    return cuda_check(cudaGetLastError(), "render");
}

// Single-instance scenes: every form the autotuner times.
template <int M>
int32_t launch_flat(uint32_t kernel, const RenderLaunch& L) {
    switch (kernel) {
        case PHX_KERNEL_STATE_MACHINE: return launch_sm<M, 4>(L);
        case PHX_KERNEL_STATE_MACHINE_6: return launch_sm<M, 6>(L);
        case PHX_KERNEL_STATE_MACHINE_8: return launch_sm<M, 8>(L);
        case PHX_KERNEL_MEGAKERNEL_3: return launch_mk<M, 3, false>(L);
        case PHX_KERNEL_MEGAKERNEL_2: return launch_mk<M, 2, false>(L);
        case PHX_KERNEL_MEGAKERNEL_SYNC: return launch_mk<M, 4, true>(L);
        case PHX_KERNEL_MEGAKERNEL_2_SYNC: return launch_mk<M, 2, true>(L);
        case PHX_KERNEL_MEGAKERNEL_5: return launch_mk<M, 5, false>(L);
        case PHX_KERNEL_MEGAKERNEL_6: return launch_mk<M, 6, false>(L);
        case PHX_KERNEL_MEGAKERNEL_6_SYNC: return launch_mk<M, 6, true>(L);
        case PHX_KERNEL_MEGAKERNEL_8: return launch_mk<M, 8, false>(L);
        case PHX_KERNEL_MEGAKERNEL_8_SYNC: return launch_mk<M, 8, true>(L);
        case PHX_KERNEL_MEGAKERNEL_10_SYNC: return launch_mk<M, 10, true>(L);
        case PHX_KERNEL_MEGAKERNEL_12_SYNC: return launch_mk<M, 12, true>(L);
        case PHX_KERNEL_MEGAKERNEL_16_SYNC: return launch_mk<M, 16, true>(L);
        default: return launch_mk<M, 4, false>(L);
    }
}


// The wavefront render: each pass runs the logic kernel over every path
// slot, then walks the primary, extension and shadow queues; the host reads
// the queue lengths every fourth pass and stops once a pass queued nothing
// (every slot is done). Passes are bounded: no more than every sample of
// every pixel a slot takes could need (1,024 rays a sample), else the
// render fails with PHX_ERR_KERNEL.
template <int M>
int32_t launch_wf(const RenderLaunch& L, const WfBuffers& B) {
    cudaStream_t s = L.s;
    const uint32_t nslots = B.nslots;
    uint32_t* words = B.words;
    float4* rays = B.rays;
    float4* hits = B.hits;
    uint32_t* hinst = B.hinst;
    uint32_t* queues = B.queues;
    uint32_t* lens = B.lens;
    const uint32_t blocks = ceil_div(nslots, 128);
    k_wf_init<<<blocks, 128, 0, s>>>(words, nslots);
    PHX_CUDA(cudaMemsetAsync(L.next, 0, 4, s));
    const uint64_t per_slot = ((uint64_t)L.count + nslots - 1) / nslots * std::max<uint32_t>(L.F.spp, 1u);
    const uint64_t limit = per_slot * 1024u + 64u;
    for (uint64_t it = 0;; it++) {
        if (it > limit) return fail(PHX_ERR_KERNEL, "wavefront render did not finish in %llu passes",
                                    (unsigned long long)limit);
        PHX_CUDA(cudaMemsetAsync(lens, 0, 12, s));
        k_wf_logic<M><<<blocks, 128, 0, s>>>(L.S, L.F, L.sun, L.px, L.first, L.count, L.next, words, nslots, hits,
                                              hinst, rays, queues, lens);
        k_wf_walk<false, M><<<blocks, 128, 0, s>>>(L.S, queues + (size_t)Q_PRIMARY * nslots, lens + Q_PRIMARY, rays,
                                                   hits, hinst, L.counters);
        k_wf_walk<false, M><<<blocks, 128, 0, s>>>(L.S, queues + (size_t)Q_EXTEND * nslots, lens + Q_EXTEND, rays,
                                                   hits, hinst, L.counters);
        k_wf_walk<true, M><<<blocks, 128, 0, s>>>(L.S, queues + (size_t)Q_SHADOW * nslots, lens + Q_SHADOW, rays,
                                                  hits, hinst, L.counters);
        PHX_CUDA(cudaGetLastError());
        if ((it & 3u) == 3u) {
            PHX_CUDA(cudaMemcpyAsync(B.host_lens, lens, 12, cudaMemcpyDeviceToHost, s));
            PHX_TRY(wait_stream(s, 0));
            if (B.host_lens[0] + B.host_lens[1] + B.host_lens[2] == 0u) break;
        }
    }
    return PHX_OK;
}

// Scenes of instances and frames with the floor grid: three forms — the
// state machine, and the megakernel at the 4-block and the 16-block
// (per-sample wait) budgets —
// each kernel id taking the one nearest its own (every form computes the
// same image).
template <int M>
int32_t launch_placed(uint32_t kernel, const RenderLaunch& L) {
    if (kernel >= PHX_KERNEL_STATE_MACHINE && kernel <= PHX_KERNEL_STATE_MACHINE_8) return launch_sm<M, 4>(L);
    if ((kernel >= PHX_KERNEL_MEGAKERNEL_8 && kernel <= PHX_KERNEL_MEGAKERNEL_16_SYNC) ||
        kernel == PHX_KERNEL_MEGAKERNEL_8_SYNC_REG || kernel == PHX_KERNEL_MEGAKERNEL_16_SYNC_REG)
        return launch_mk<M, 16, true>(L);
    return launch_mk<M, 4, false>(L);
}


}  // namespace
}  // namespace phx
