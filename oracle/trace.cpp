// ORACLE — test infrastructure only (see oracle.h). CPU restatement of
// phiray's Rendered-mode path tracer: src/trace/wgsl/shade.wgsl main,
// integrate.wgsl, light.wgsl, brdf.wgsl, bvh.wgsl, util.wgsl, view.wgsl and
// layout.wgsl, over a scene of one identity instance whose tree is the
// oracle's own Bvh::build (leaf order = the faces reordered by `order`, as
// Scene::reorder does, src/trace/build.rs:147). The emitter table follows
// lamp.rs table_of. Each sample is accumulated into the px buffer the way
// util.wgsl's emit and guide do (read-modify-write per sample).
//
// Only the features the synthetic configs use are restated; the rest
// (textures, procedural slots, environment images, depth of field, film
// transparency, other pixel filters and view transforms) must be off in the
// Camera.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/phiray_cuda.h"
#include "oracle.h"
#include "wgsl.h"

using namespace wg;

namespace {

const uint32_t LEAF = 0x80000000u;
const uint32_t NONE = 0xffffffffu;
const float INF = 3.0e38f;
const float PI = 3.14159265f;

struct Hit {
    float t;
    uint32_t tri;  // slot (face in leaf order)
    float u, v;
    uint32_t inst;
};

// A triangle record as layout.wgsl's tri_of assembles it.
struct Tri {
    V3 a, b, c, na, nb, nc;
    bool mirror;  // placed by an instance whose matrix mirrors (word 27, bit 2)
    float rough, trans, metal, ior;
    float color[4];
    V3 emit;
    float sss;
    V3 sss_radius;
    float sheen, sheen_rough;
    V3 sheen_tint;
    float coat, coat_rough;
};

struct Surf {
    V3 pos, n, v, albedo, f0;
    float rough, bleed;
    V3 sss_tint;
    float sheen, sheen_rough;
    V3 sheen_tint;
    float coat, coat_rough, eta, dielectric;
};

struct Shadowed {
    V3 c, dir;
    float dist;
};

// One placement of a mesh (instance.rs Instance::words): the world matrix's
// rows, the inverse's rows, the mesh, and flags — bit 0 at the identity,
// bit 1 casts no shadow, bit 2 mirrors.
struct Inst {
    float row[3][4];
    float inv[3][4];
    uint32_t mesh;
    uint32_t flags;
};

// One mesh's tree (forest.rs blas): faces [lo, hi) of the scene, nodes over
// them in the mesh's own space, leaf ranges mesh-local.
struct MeshTree {
    uint32_t lo = 0, hi = 0;
    std::vector<orc_node> nodes;
};

// The scene shared by every pixel: the tree, leaf order, emitter table.
// With `meshes` empty the scene is one identity instance whose tree is
// `nodes`; otherwise `nodes` is the top tree over the instances' world boxes
// (its slots named by inst_order) and each mesh has its own tree.
struct Shared {
    std::vector<orc_node> nodes;
    std::vector<uint32_t> order;
    std::vector<uint32_t> lamp_face;  // light table (lamp.rs table_of): slots
    std::vector<uint32_t> lamp_inst;  // and the instance of each
    std::vector<float> lamp_cdf;
    float extent = 0.0f;
    std::vector<MeshTree> meshes;
    std::vector<Inst> insts;
    std::vector<uint32_t> inst_order;
    uint32_t leaf = 4;
};

struct World {
    const Shared* S = nullptr;
    const float* verts;
    const float* normals;
    const uint32_t* faces;  // original order
    const float* mats;
    const phx_camera* p;
    uint32_t n, frame;
    float ao, eps;
    uint32_t* px;
    uint64_t rays;
    mutable uint64_t steps = 0, tests = 0;  // inner-node visits and triangle tests of the walks

    const uint32_t* face(uint32_t slot) const { return faces + 4 * (size_t)S->order[slot]; }
    V3 vert(uint32_t v) const { return v3(verts[4 * (size_t)v], verts[4 * (size_t)v + 1], verts[4 * (size_t)v + 2]); }
    const float* mat(uint32_t m) const { return mats + 32 * (size_t)m; }
};

// util.wgsl:1-10
uint32_t hash(uint32_t x) {
    uint32_t h = x * 747796405u + 2891336453u;
    h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
    return (h >> 22u) ^ h;
}
float rnd(uint32_t* seed) {
    *seed = hash(*seed);
    return (float)*seed / 4294967295.0f;
}

// util.wgsl unit_disk
void unit_disk(float ru, float rv, float* ox, float* oy) {
    const float a = 2.0f * ru - 1.0f;
    const float b = 2.0f * rv - 1.0f;
    if (a == 0.0f && b == 0.0f) {
        *ox = 0.0f;
        *oy = 0.0f;
        return;
    }
    float r, phi;
    if (a * a > b * b) {
        r = a;
        phi = (PI / 4.0f) * (b / a);
    } else {
        r = b;
        phi = (PI / 2.0f) - (PI / 4.0f) * (a / b);
    }
    *ox = r * pm_cos(phi);
    *oy = r * pm_sin(phi);
}

// ---- bvh.wgsl ----

float box_t(const orc_node& nd, V3 o, V3 inv, float best) {
    const V3 lo = v3(nd.lo.p[0], nd.lo.p[1], nd.lo.p[2]), hi = v3(nd.hi.p[0], nd.hi.p[1], nd.hi.p[2]);
    const V3 t1 = (lo - o) * inv;
    const V3 t2 = (hi - o) * inv;
    const float tmin = fmaxw(fmaxw(fminw(t1.x, t2.x), fminw(t1.y, t2.y)), fminw(t1.z, t2.z));
    const float tmax = fminw(fminw(fmaxw(t1.x, t2.x), fmaxw(t1.y, t2.y)), fmaxw(t1.z, t2.z));
    if (tmax >= fmaxw(tmin, 0.0f) && tmin < best) return fmaxw(tmin, 0.0f);
    return INF;
}

struct RaySpace {
    uint32_t kz;
    bool flip;
    V3 s;
};

V3 ray_axes(V3 v, uint32_t kz, bool flip) {
    V3 p = v;
    if (kz == 0u) p = v3(v.y, v.z, v.x);
    else if (kz == 1u) p = v3(v.z, v.x, v.y);
    if (flip) p = v3(p.y, p.x, p.z);
    return p;
}

RaySpace ray_space(V3 d) {
    const V3 a = vabs(d);
    uint32_t kz = 2u;
    if (a.x >= a.y && a.x >= a.z) kz = 0u;
    else if (a.y >= a.z) kz = 1u;
    const bool flip = ray_axes(d, kz, false).z < 0.0f;
    const V3 dr = ray_axes(d, kz, flip);
    const float sz = 1.0f / dr.z;
    return RaySpace{kz, flip, v3(dr.x * sz, dr.y * sz, sz)};
}

// tri_t: (t, u, v) or t = INF
void tri_t(V3 ta, V3 tb, V3 tc, V3 o, const RaySpace& r, float out[3]) {
    out[0] = INF;
    out[1] = out[2] = 0.0f;
    const V3 a = ray_axes(ta - o, r.kz, r.flip);
    const V3 b = ray_axes(tb - o, r.kz, r.flip);
    const V3 c = ray_axes(tc - o, r.kz, r.flip);
    const float ax = a.x - r.s.x * a.z;
    const float ay = a.y - r.s.y * a.z;
    const float bx = b.x - r.s.x * b.z;
    const float by = b.y - r.s.y * b.z;
    const float cx = c.x - r.s.x * c.z;
    const float cy = c.y - r.s.y * c.z;
    const float ea = cx * by - cy * bx;
    const float eb = ax * cy - ay * cx;
    const float ec = bx * ay - by * ax;
    if ((ea < 0.0f || eb < 0.0f || ec < 0.0f) && (ea > 0.0f || eb > 0.0f || ec > 0.0f)) return;
    const float det = ea + eb + ec;
    if (det == 0.0f) return;
    const float tt = ea * (r.s.z * a.z) + eb * (r.s.z * b.z) + ec * (r.s.z * c.z);
    const float sg = det < 0.0f ? -1.0f : 1.0f;
    if (tt * sg <= 0.0f) return;
    const float inv = 1.0f / det;
    out[0] = tt * inv;
    out[1] = eb * inv;
    out[2] = ec * inv;
}

V3 safe_inv(V3 d) {
    const V3 s = v3(d.x < 0.0f ? -1.0f : 1.0f, d.y < 0.0f ? -1.0f : 1.0f, d.z < 0.0f ? -1.0f : 1.0f);
    const V3 q = v3(std::fabs(d.x) < 1e-9f ? s.x * 1e-9f : d.x, std::fabs(d.y) < 1e-9f ? s.y * 1e-9f : d.y,
                    std::fabs(d.z) < 1e-9f ? s.z * 1e-9f : d.z);
    return v3(1.0f / q.x, 1.0f / q.y, 1.0f / q.z);
}

// trace_blas (bvh.wgsl:120-190) for the single identity instance.
void trace_blas(const World& W, V3 o, V3 d, bool first, Hit* best) {
    const V3 inv = safe_inv(d);
    const orc_node top = W.S->nodes[0];
    if (box_t(top, o, inv, best->t) >= INF) return;
    const RaySpace rs = ray_space(d);
    uint32_t stack[32];
    uint32_t sp = 0;
    orc_node nd = top;
    for (;;) {
        if ((nd.lo.i & LEAF) != 0u) {
            for (uint32_t id = nd.lo.i & ~LEAF; id < nd.hi.i; id++) {
                const uint32_t* v = W.face(id);
                W.tests++;
                float h[3];
                tri_t(W.vert(v[0]), W.vert(v[1]), W.vert(v[2]), o, rs, h);
                if (h[0] < best->t) {
                    if (first) {
                        const float* m = W.mat(v[3]);
                        if (m[6] > 0.5f || m[3] < 0.5f) continue;
                        *best = Hit{h[0], id, h[1], h[2], 0};
                        return;
                    }
                    *best = Hit{h[0], id, h[1], h[2], 0};
                }
            }
        } else {
            W.steps++;
            const orc_node nl = W.S->nodes[nd.lo.i];
            const orc_node nr = W.S->nodes[nd.hi.i];
            const float tl = box_t(nl, o, inv, best->t);
            const float tr = box_t(nr, o, inv, best->t);
            if (tl < INF && tr < INF) {
                if (tl <= tr) {
                    stack[sp] = nd.hi.i;
                    nd = nl;
                } else {
                    stack[sp] = nd.lo.i;
                    nd = nr;
                }
                sp++;
                continue;
            }
            if (tl < INF) {
                nd = nl;
                continue;
            }
            if (tr < INF) {
                nd = nr;
                continue;
            }
        }
        if (sp == 0u) break;
        sp--;
        nd = W.S->nodes[stack[sp]];
    }
}

// A row of an instance matrix applied to a point (w = 1) or a direction.
float row_point(const float r[4], V3 p) { return ((r[0] * p.x + r[1] * p.y) + r[2] * p.z) + r[3] * 1.0f; }
float row_dir(const float r[4], V3 d) { return (r[0] * d.x + r[1] * d.y) + r[2] * d.z; }

// trace_blas (bvh.wgsl:115-190) for instance i of a scene with a top tree:
// the ray taken into the mesh's space by the instance's inverse (direction
// unnormalised, so t is the world's), the mesh's tree walked there.
void trace_blas_inst(const World& W, uint32_t i, V3 ow, V3 dw, bool first, Hit* best) {
    const Inst& in = W.S->insts[i];
    const MeshTree& mt = W.S->meshes[in.mesh];
    if (mt.nodes.empty()) return;
    if (first && (in.flags & 2u) != 0u) return;
    V3 o = ow, d = dw;
    if ((in.flags & 1u) == 0u) {
        o = v3(row_point(in.inv[0], ow), row_point(in.inv[1], ow), row_point(in.inv[2], ow));
        d = v3(row_dir(in.inv[0], dw), row_dir(in.inv[1], dw), row_dir(in.inv[2], dw));
    }
    const V3 inv = safe_inv(d);
    const orc_node top = mt.nodes[0];
    if (box_t(top, o, inv, best->t) >= INF) return;
    const RaySpace rs = ray_space(d);
    uint32_t stack[32];
    uint32_t sp = 0;
    orc_node nd = top;
    for (;;) {
        if ((nd.lo.i & LEAF) != 0u) {
            for (uint32_t id = (nd.lo.i & ~LEAF) + mt.lo; id < nd.hi.i + mt.lo; id++) {
                const uint32_t* v = W.face(id);
                W.tests++;
                float h[3];
                tri_t(W.vert(v[0]), W.vert(v[1]), W.vert(v[2]), o, rs, h);
                if (h[0] < best->t) {
                    if (first) {
                        const float* m = W.mat(v[3]);
                        if (m[6] > 0.5f || m[3] < 0.5f) continue;
                        *best = Hit{h[0], id, h[1], h[2], i};
                        return;
                    }
                    *best = Hit{h[0], id, h[1], h[2], i};
                }
            }
        } else {
            W.steps++;
            const orc_node nl = mt.nodes[nd.lo.i];
            const orc_node nr = mt.nodes[nd.hi.i];
            const float tl = box_t(nl, o, inv, best->t);
            const float tr = box_t(nr, o, inv, best->t);
            if (tl < INF && tr < INF) {
                if (tl <= tr) {
                    stack[sp] = nd.hi.i;
                    nd = nl;
                } else {
                    stack[sp] = nd.lo.i;
                    nd = nr;
                }
                sp++;
                continue;
            }
            if (tl < INF) {
                nd = nl;
                continue;
            }
            if (tr < INF) {
                nd = nr;
                continue;
            }
        }
        if (sp == 0u) break;
        sp--;
        nd = mt.nodes[stack[sp]];
    }
}

// trace (bvh.wgsl:194-232). One identity instance: its tree is `nodes`.
// With instances: the top tree over their world boxes, each leaf's
// instances walked in slot order; an any-hit ray stops at the first.
Hit trace(World& W, V3 o, V3 d, float tmax, bool first) {
    W.rays++;
    Hit best{tmax, NONE, 0.0f, 0.0f, 0};
    const V3 inv = safe_inv(d);
    if (W.S->nodes.empty() || box_t(W.S->nodes[0], o, inv, best.t) >= INF) return best;
    if (W.S->meshes.empty()) {
        trace_blas(W, o, d, first, &best);
        return best;
    }
    uint32_t stack[32];
    uint32_t sp = 0;
    orc_node nd = W.S->nodes[0];
    for (;;) {
        if ((nd.lo.i & LEAF) != 0u) {
            for (uint32_t s = nd.lo.i & ~LEAF; s < nd.hi.i; s++) {
                trace_blas_inst(W, W.S->inst_order[s], o, d, first, &best);
                if (first && best.tri != NONE) return best;
            }
        } else {
            W.steps++;
            const orc_node nl = W.S->nodes[nd.lo.i];
            const orc_node nr = W.S->nodes[nd.hi.i];
            const float tl = box_t(nl, o, inv, best.t);
            const float tr = box_t(nr, o, inv, best.t);
            if (tl < INF && tr < INF) {
                if (tl <= tr) {
                    stack[sp] = nd.hi.i;
                    nd = nl;
                } else {
                    stack[sp] = nd.lo.i;
                    nd = nr;
                }
                sp++;
                continue;
            }
            if (tl < INF) {
                nd = nl;
                continue;
            }
            if (tr < INF) {
                nd = nr;
                continue;
            }
        }
        if (sp == 0u) break;
        sp--;
        nd = W.S->nodes[stack[sp]];
    }
    return best;
}

float visible(World& W, V3 org, V3 l, float dist) { return trace(W, org, l, dist, true).tri != NONE ? 0.0f : 1.0f; }

// ---- layout.wgsl ----

// place_n (layout.wgsl:72-77): a normal under the inverse-transpose of an
// instance's 3 x 3, unit again; a zero (flat) normal stays zero.
V3 place_n(const Inst& in, V3 n) {
    const V3 m = v3(in.inv[0][0], in.inv[0][1], in.inv[0][2]) * n.x + v3(in.inv[1][0], in.inv[1][1], in.inv[1][2]) * n.y +
                 v3(in.inv[2][0], in.inv[2][1], in.inv[2][2]) * n.z;
    const float l = length(m);
    if (l < 1e-12f) return v3(0.0f);
    return m / l;
}

// tri_of (layout.wgsl:114-159): the face in slot `slot`, placed in the world
// by instance `inst` (its vertices are kept in the mesh's space).
Tri tri_of(const World& W, uint32_t slot, uint32_t inst = 0) {
    const uint32_t* v = W.face(slot);
    const float* m = W.mat(v[3]);
    Tri t;
    t.a = W.vert(v[0]);
    t.b = W.vert(v[1]);
    t.c = W.vert(v[2]);
    t.mirror = false;
    if (W.normals) {
        auto nv = [&](uint32_t k) {
            return v3(W.normals[4 * (size_t)k], W.normals[4 * (size_t)k + 1], W.normals[4 * (size_t)k + 2]);
        };
        t.na = nv(v[0]);
        t.nb = nv(v[1]);
        t.nc = nv(v[2]);
    } else {
        t.na = t.nb = t.nc = v3(0.0f);
    }
    if (!W.S->insts.empty()) {
        const Inst& in = W.S->insts[inst];
        t.mirror = (in.flags & 4u) != 0u;
        if ((in.flags & 1u) == 0u) {
            auto place = [&](uint32_t k) {  // the vertex with w = 1, as the scene stores it
                const float* q = W.verts + 4 * (size_t)k;
                auto r = [&](const float* row) { return ((row[0] * q[0] + row[1] * q[1]) + row[2] * q[2]) + row[3]; };
                return v3(r(in.row[0]), r(in.row[1]), r(in.row[2]));
            };
            t.a = place(v[0]);
            t.b = place(v[1]);
            t.c = place(v[2]);
            t.na = place_n(in, t.na);
            t.nb = place_n(in, t.nb);
            t.nc = place_n(in, t.nc);
        }
    }
    t.rough = m[4];
    t.metal = m[5];
    t.trans = m[6];
    t.ior = m[7];
    for (int k = 0; k < 4; k++) t.color[k] = m[k];
    t.emit = v3(m[8], m[9], m[10]);
    t.sss = m[17];
    t.sss_radius = v3(m[18], m[19], m[20]);
    t.sheen = m[21];
    t.sheen_rough = m[22];
    t.sheen_tint = v3(m[23], m[24], m[25]);
    t.coat = m[26];
    t.coat_rough = m[27];
    return t;
}

// world_ng (layout.wgsl:97-101): turned back under a mirroring instance.
V3 world_ng(const Tri& t) {
    const V3 ng = normalize(cross(t.b - t.a, t.c - t.a));
    return t.mirror ? -ng : ng;
}

// ---- brdf.wgsl ----

float ggx_lambda(float alpha2, float cos_n) {
    const float t = alpha2 * fmaxw(1.0f / fmaxw(cos_n * cos_n, 1e-8f) - 1.0f, 0.0f);
    return 0.5f * (std::sqrt(1.0f + t) - 1.0f);
}

V3 ggx_sample_vndf(V3 wi, float alpha, float r1, float r2) {
    const V3 wi_ = normalize(v3(alpha * wi.x, alpha * wi.y, wi.z));
    const float lensq = wi_.x * wi_.x + wi_.y * wi_.y;
    V3 t1, t2;
    if (lensq > 1e-7f) {
        t1 = v3(-wi_.y, wi_.x, 0.0f) / std::sqrt(lensq);
        t2 = cross(wi_, t1);
    } else {
        t1 = v3(1.0f, 0.0f, 0.0f);
        t2 = v3(0.0f, 1.0f, 0.0f);
    }
    float tx, ty;
    unit_disk(r1, r2, &tx, &ty);
    ty = mixf(std::sqrt(fmaxw(1.0f - tx * tx, 0.0f)), ty, 0.5f * (1.0f + wi_.z));
    const V3 h_ = t1 * tx + t2 * ty + wi_ * std::sqrt(fmaxw(0.0f, 1.0f - tx * tx - ty * ty));
    return normalize(v3(alpha * h_.x, alpha * h_.y, fmaxw(0.0f, h_.z)));
}

float ggx_weight(float alpha2, float cos_ni, float cos_no) {
    const float li = ggx_lambda(alpha2, cos_ni);
    const float lo = ggx_lambda(alpha2, cos_no);
    return (1.0f + li) / (1.0f + li + lo);
}

Surf plain_surf(V3 pos, V3 n, V3 v, V3 albedo, V3 f0, float rough) {
    return Surf{pos, n, v, albedo, f0, rough, 0.0f, v3(1.0f), 0.0f, 0.5f, v3(1.0f), 0.0f, 0.03f, 0.0f, 0.0f};
}

float fresnel_dielectric_cos(float cosi, float eta) {
    const float c = std::fabs(cosi);
    float g = eta * eta - 1.0f + c * c;
    if (g <= 0.0f) return 1.0f;
    g = std::sqrt(g);
    const float a = (g - c) / (g + c);
    const float b = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
    return 0.5f * a * a * (1.0f + b * b);
}

V3 fresnel_of(const Surf& s, float cs) {
    const float schlick = pm_pow(1.0f - cs, 5.0f);
    V3 f = s.f0 + (v3(1.0f) - s.f0) * schlick;
    if (s.eta > 1.0f && s.dielectric > 0.0f) {
        const float r = (s.eta - 1.0f) / (s.eta + 1.0f);
        const float face_on = r * r;
        f += v3(s.dielectric * (fresnel_dielectric_cos(cs, s.eta) - face_on - (1.0f - face_on) * schlick));
    }
    return vmax(f, v3(0.0f));
}

V3 scatter_tint(V3 radius) {
    const float m = fmaxw(fmaxw(radius.x, radius.y), fmaxw(radius.z, 1e-6f));
    return vmix(v3(1.0f), radius / m, 0.85f);
}

float scatter_bleed(float weight, V3 radius) {
    const float m = fmaxw(fmaxw(radius.x, radius.y), fmaxw(radius.z, 0.0f));
    return clampf(weight, 0.0f, 1.0f) * clampf(m * 24.0f, 0.15f, 1.0f);
}

float charlie(float nh, float rough) {
    const float inv = 1.0f / fmaxw(rough * rough, 0.005f);
    const float sin2 = fmaxw(1.0f - nh * nh, 0.0f);
    return (2.0f + inv) * pm_pow(sin2, inv * 0.5f) / (2.0f * PI);
}

V3 env_brdf(V3 f0, float rough, float nv) {
    const float c0[4] = {-1.0f, -0.0275f, -0.572f, 0.022f};
    const float c1[4] = {1.0f, 0.0425f, 1.04f, -0.04f};
    float r[4];
    for (int k = 0; k < 4; k++) r[k] = rough * c0[k] + c1[k];
    const float a004 = fminw(r[0] * r[0], pm_exp2(-9.28f * nv)) * r[0] + r[1];
    const float abx = -1.04f * a004 + r[2];
    const float aby = 1.04f * a004 + r[3];
    return f0 * abx + v3(aby);
}

V3 dielectric_f0(float ior) {
    const float r = (ior - 1.0f) / (ior + 1.0f);
    return v3(r * r);
}

float under_layer(V3 f0, float rough, float nv) {
    const V3 e = env_brdf(f0, rough, nv);
    return clampf(1.0f - maxc(e), 0.0f, 1.0f);
}

float under_layer_real(float eta, float rough, float nv) {
    const float r = (eta - 1.0f) / (eta + 1.0f);
    const float face_on = r * r;
    const float climb = env_brdf(v3(0.0f), rough, nv).x;
    const float flat = env_brdf(v3(1.0f), rough, nv).x - climb;
    const float schlick = (1.0f - face_on) * pm_pow(1.0f - nv, 5.0f);
    const float real = fresnel_dielectric_cos(nv, eta) - face_on;
    const float scale = clampf(real / fmaxw(schlick, 1e-5f), 0.0f, 1.0f);
    return clampf(1.0f - (face_on * flat + climb * scale), 0.0f, 1.0f);
}

// brdf.wgsl glossy_floor, phiray's own integrator (integrator.x = 0).
float glossy_floor(float) { return 0.3f; }

float ggx_pdf(const Surf& s, V3 l) {
    const V3 h = normalize(l + s.v);
    const float nh = fmaxw(dot(s.n, h), 0.0f);
    const float a2 = fmaxw(s.rough * s.rough * s.rough * s.rough, 1e-4f);
    const float dd = nh * nh * (a2 - 1.0f) + 1.0f;
    const float dist = a2 / (PI * dd * dd);
    const float nv = fmaxw(dot(s.n, s.v), 1e-4f);
    const float g1 = 1.0f / (1.0f + ggx_lambda(a2, nv));
    return g1 * dist / (4.0f * nv);
}

// brdf_w (brdf.wgsl:231-269). The subsurface, sheen and coat terms are
// evaluated only when their weight is non-zero: each is a product with that
// weight, so a zero weight contributes exactly zero.
V3 brdf_w(const Surf& s, V3 l, V3 e, float wd, float ws) {
    const float raw = dot(s.n, l);
    const float w = s.bleed * 0.75f;
    const float nl = fmaxw((raw + w) / (1.0f + w), 0.0f) / (1.0f + w * 0.5f);
    V3 thru = v3(0.0f);
    if (s.bleed != 0.0f) thru = s.bleed * s.albedo * s.sss_tint * pm_pow(fmaxw(dot(s.v, -l), 0.0f), 3.0f) * 0.35f;
    if (nl <= 0.0f) return thru * e * wd;
    const V3 hv = normalize(l + s.v);
    const float nh = fmaxw(dot(s.n, hv), 0.0f);
    const float hvv = fmaxw(dot(hv, s.v), 0.0f);
    const float a2 = fmaxw(s.rough * s.rough * s.rough * s.rough, 1e-4f);
    const float dd = nh * nh * (a2 - 1.0f) + 1.0f;
    const float dist = a2 / (PI * dd * dd);
    const V3 fres = fresnel_of(s, hvv);
    const float nv = fmaxw(dot(s.n, s.v), 1e-4f);
    const float g2 = 1.0f / (1.0f + ggx_lambda(a2, nv) + ggx_lambda(a2, fmaxw(raw, 1e-4f)));
    const V3 spec = fres * dist * g2 * 0.25f / nv;
    const V3 diffuse = vmix(s.albedo, s.albedo * s.sss_tint, s.bleed) / PI;
    V3 sum = diffuse * wd + spec * ws;
    if (s.sheen != 0.0f) sum += s.sheen * s.sheen_tint * charlie(nh, s.sheen_rough);
    if (s.coat != 0.0f) {
        const float ca2 = fmaxw(s.coat_rough * s.coat_rough * s.coat_rough * s.coat_rough, 1e-4f);
        const float cd = nh * nh * (ca2 - 1.0f) + 1.0f;
        const float coat_f = 0.04f + 0.96f * pm_pow(1.0f - hvv, 5.0f);
        const float coat = s.coat * coat_f * (ca2 / (PI * cd * cd)) * 0.25f;
        const float under = 1.0f - s.coat * coat_f;
        sum = sum * under + v3(coat);
    }
    V3 out = sum * e * nl;
    if (s.bleed != 0.0f) out += thru * e * wd;
    return out;
}

V3 brdf(const Surf& s, V3 l, V3 e) { return brdf_w(s, l, e, 1.0f, 1.0f); }

// ---- light.wgsl ----

V3 onb(V3 n, float a, float b) {
    const V3 tx = normalize(std::fabs(n.z) > 0.9f ? cross(n, v3(1.0f, 0.0f, 0.0f)) : cross(n, v3(0.0f, 0.0f, 1.0f)));
    const V3 ty = cross(n, tx);
    return tx * a + ty * b;
}

float spot_mask(const phx_light& li, V3 l) {
    const V3 dir = v3(li.dir[0], li.dir[1], li.dir[2]);
    const V3 right = v3(li.right[0], li.right[1], li.right[2]);
    const float z = -dot(l, dir);
    if (z <= 0.0f) return 0.0f;
    float ellipse = z;
    if (dot(right, right) > 1e-12f &&
        li.spot_scale[0] * li.spot_scale[0] + li.spot_scale[1] * li.spot_scale[1] > 1e-12f) {
        const V3 d = -l;
        const float x = dot(d, right) * li.spot_scale[0];
        const float y = dot(d, cross(dir, right)) * li.spot_scale[1];
        ellipse = 1.0f / std::sqrt(1.0f + (x * x + y * y) / (z * z));
    }
    return smoothstep(li.cone, li.cone + li.blend, ellipse);
}

V3 cone_dir(V3 axis, float ang, uint32_t* seed) {
    if (ang <= 0.0f) return axis;
    const float r = ang * std::sqrt(rnd(seed));
    const float ph = 2.0f * PI * rnd(seed);
    return normalize(axis + onb(axis, r * pm_cos(ph), r * pm_sin(ph)));
}

V3 env_at(const World& W, V3) { return v3(W.p->env[0], W.p->env[1], W.p->env[2]); }

Shadowed unshadowed() { return Shadowed{v3(0.0f), v3(0.0f, 0.0f, 1.0f), 0.0f}; }

bool uses_rig(const World& W) {
    const V3 env = v3(W.p->env[0], W.p->env[1], W.p->env[2]);
    const bool world_lit = W.p->envmap != 0u || dot(env, env) > 0.0f;
    return W.p->count == 0u && !world_lit;
}

V3 vec(const float* f) { return v3(f[0], f[1], f[2]); }

Shadowed rig_query(const World& W, uint32_t k, const Surf& s, uint32_t* seed) {
    if (k == 0u) {
        const V3 key = cone_dir(vec(W.p->sun), 0.06f, seed);
        return Shadowed{brdf(s, key, v3(2.0f)), key, INF};
    }
    const V3 rim = normalize(vec(W.p->up) * 0.6f - vec(W.p->back) * 0.8f + vec(W.p->right) * 0.2f);
    return Shadowed{brdf(s, rim, v3(0.9f)), rim, INF};
}

V3 rig_fill(const World& W, const Surf& s) {
    const V3 fill = normalize(-vec(W.p->right) * 0.8f + vec(W.p->up) * 0.2f + vec(W.p->back) * 0.6f);
    return brdf(s, fill, v3(0.45f));
}

float lamp_reach(const World& W, const phx_light& li, V3 at) {
    const float lum = dot(vmax(vec(li.color), v3(0.0f)), v3(0.2126f, 0.7152f, 0.0722f));
    if (li.kind == 0u) return lum;
    const V3 to = vec(li.pos) - at;
    const float near = fmaxw(li.size * 0.5f, W.ao * 0.05f);
    return lum / (4.0f * PI * (dot(to, to) + near * near));
}

Shadowed area_query(const Surf& s, const phx_light& li, float weight, float r1, float r2, float pick) {
    const V3 lpos = vec(li.pos), ldir = vec(li.dir), lright = vec(li.right);
    const float height = dot(s.pos - lpos, ldir);
    if (height <= 0.0f) return unshadowed();
    const bool round = li.shape == 4u || li.shape == 5u;
    const float half[2] = {li.size * 0.5f, li.size_y * 0.5f};
    const float area = fmaxw(li.size * li.size_y * (round ? 0.25f * PI : 1.0f), 1e-8f);
    const V3 up = cross(ldir, lright);
    const V3 off = s.pos - lpos;
    const float near = area / (area + PI * dot(off, off));
    float on[2];
    if (pick < near) {
        const float spread = std::sqrt(r1 / fmaxw(1.0f - r1, 1e-6f)) * height;
        on[0] = pm_cos(2.0f * PI * r2) * spread + dot(off, lright);
        on[1] = pm_sin(2.0f * PI * r2) * spread + dot(off, up);
        const float unit[2] = {on[0] / fmaxw(half[0], 1e-8f), on[1] / fmaxw(half[1], 1e-8f)};
        const bool inside = round ? (unit[0] * unit[0] + unit[1] * unit[1] <= 1.0f)
                                  : (fmaxw(std::fabs(unit[0]), std::fabs(unit[1])) <= 1.0f);
        if (!inside) return unshadowed();
    } else {
        const float disk[2] = {pm_cos(2.0f * PI * r2) * std::sqrt(r1), pm_sin(2.0f * PI * r2) * std::sqrt(r1)};
        if (round) {
            on[0] = disk[0] * half[0];
            on[1] = disk[1] * half[1];
        } else {
            on[0] = (r1 * 2.0f - 1.0f) * half[0];
            on[1] = (r2 * 2.0f - 1.0f) * half[1];
        }
    }
    const V3 to = lpos + lright * on[0] + up * on[1] - s.pos;
    const float d2 = fmaxw(dot(to, to), 1e-6f);
    const V3 l = to / std::sqrt(d2);
    const float facing = fmaxw(dot(-l, ldir), 0.0f);
    const float pdf = (1.0f - near) / area + near * facing * facing / (PI * d2);
    const V3 e = vec(li.color) / (PI * area) * facing / d2 / fmaxw(pdf, 1e-12f);
    if (maxc(e) < 1e-5f) return unshadowed();
    return Shadowed{brdf(s, l, e) * weight, l, std::sqrt(d2) * 0.999f};
}

Shadowed lamp_query(const World& W, const Surf& s, uint32_t* seed) {
    float total = 0.0f;
    uint32_t idx = 0;
    float held = 0.0f;
    float u = rnd(seed);
    for (uint32_t k = 0; k < W.p->count; k++) {
        const float w = lamp_reach(W, W.p->lights[k], s.pos);
        if (w <= 0.0f) continue;
        total += w;
        const float share = w / total;
        if (u < share) {
            idx = k;
            held = w;
            u = u / share;
        } else {
            u = (u - share) / (1.0f - share);
        }
    }
    if (total <= 0.0f || held <= 0.0f) return unshadowed();
    const phx_light& li = W.p->lights[idx];
    const float weight = total / held;
    if (li.kind == 0u) {
        const V3 l = cone_dir(-vec(li.dir), li.size * 0.5f, seed);
        return Shadowed{brdf(s, l, vec(li.color)) * weight, l, INF};
    }
    const float r1 = rnd(seed);
    const float r2 = rnd(seed);
    if (li.kind == 3u) return area_query(s, li, weight, r1, r2, rnd(seed));
    const V3 aim = vec(li.pos) + onb(normalize(s.pos - vec(li.pos)), (r1 - 0.5f) * li.size, (r2 - 0.5f) * li.size);
    const V3 to = aim - s.pos;
    const float d2 = fmaxw(dot(to, to), 1e-6f);
    const V3 l = to / std::sqrt(d2);
    V3 e = vec(li.color) / (4.0f * PI * d2);
    if (li.kind == 2u) e *= spot_mask(li, l);
    if (maxc(e) < 1e-5f) return unshadowed();
    return Shadowed{brdf(s, l, e) * weight, l, std::sqrt(d2) * 0.999f};
}

float hit_lift(const World& W, float t) {
    const float start = 1.0e4f / W.p->units;
    if (W.p->persp == 0u && t > start * 0.5f) return W.eps + std::fabs(t - start) * 1e-5f + start * 2.4e-7f;
    return W.eps + t * 1e-5f;
}

float through_lift(const World& W, V3 pos, float t) {
    const float reach = fmaxw(fmaxw(std::fabs(pos.x), std::fabs(pos.y)), fmaxw(std::fabs(pos.z), 0.5f));
    return hit_lift(W, t) - W.eps + reach * (256.0f / 8388608.0f);
}

// lamp_chance (light.wgsl:255-271): the share of the table a hit holds.
float lamp_chance(const World& W, const Hit& h) {
    const uint32_t count = (uint32_t)W.S->lamp_face.size();
    if (count == 0u) return 0.0f;
    uint32_t lo = 0, hi = count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2u;
        const uint32_t f = W.S->lamp_face[mid];
        const uint32_t i = W.S->lamp_inst[mid];
        if (f < h.tri || (f == h.tri && i < h.inst)) lo = mid + 1u;
        else hi = mid;
    }
    if (W.S->lamp_face[lo] != h.tri || W.S->lamp_inst[lo] != h.inst) return 0.0f;
    const float prev = lo > 0u ? W.S->lamp_cdf[lo - 1u] : 0.0f;
    return W.S->lamp_cdf[lo] - prev;
}

Shadowed glow_query(const World& W, const Surf& s, uint32_t* seed) {
    const uint32_t count = (uint32_t)W.S->lamp_face.size();
    if (count == 0u) return unshadowed();
    const float u = rnd(seed);
    uint32_t lo = 0, hi = count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2u;
        if (W.S->lamp_cdf[mid] < u) lo = mid + 1u;
        else hi = mid;
    }
    const float prev = lo > 0u ? W.S->lamp_cdf[lo - 1u] : 0.0f;
    const float chance = fmaxw(W.S->lamp_cdf[lo] - prev, 1e-8f);
    const Tri t = tri_of(W, W.S->lamp_face[lo], W.S->lamp_inst[lo]);
    float a = rnd(seed);
    float b = rnd(seed);
    if (a + b > 1.0f) {
        a = 1.0f - a;
        b = 1.0f - b;
    }
    const V3 q = t.a + (t.b - t.a) * a + (t.c - t.a) * b;
    const V3 cr = cross(t.b - t.a, t.c - t.a);
    const float area = 0.5f * length(cr);
    const V3 to = q - s.pos;
    const float d2 = fmaxw(dot(to, to), 1e-6f);
    const V3 l = to / std::sqrt(d2);
    const float cos_l = std::fabs(dot(normalize(cr), l));
    const V3 e = t.emit * cos_l * area / (chance * d2);
    const float pl = chance * d2 / fmaxw(area * cos_l, 1e-8f);
    const float pb = fmaxw(dot(s.n, l), 0.0f) / PI;
    const float w = pl * pl / fmaxw(pl * pl + pb * pb, 1e-12f);
    return Shadowed{brdf(s, l, e) * w, l, std::sqrt(d2) * 0.999f};
}

// ---- integrate.wgsl ----

V3 cosine_dir(V3 n, uint32_t* seed) {
    const float r1 = rnd(seed);
    const float rr = std::sqrt(r1);
    const float ph = 2.0f * PI * rnd(seed);
    return normalize(onb(n, rr * pm_cos(ph), rr * pm_sin(ph)) + n * std::sqrt(fmaxw(0.0f, 1.0f - r1)));
}

V3 glow_mis(const World& W, const Tri& t, const Hit& h, V3 from_n, V3 dir) {
    const V3 e = t.emit;
    const float chance = lamp_chance(W, h);
    if (chance <= 0.0f) return e;
    const V3 cr = cross(t.b - t.a, t.c - t.a);
    const float pl = chance * h.t * h.t / fmaxw(0.5f * length(cr) * std::fabs(dot(normalize(cr), dir)), 1e-8f);
    const float pb = fmaxw(dot(from_n, dir), 0.0f) / PI;
    return e * pb * pb / fmaxw(pb * pb + pl * pl, 1e-12f);
}

V3 direct(World& W, const Surf& s, uint32_t* seed, bool with_env) {
    (void)with_env;  // env_query needs an environment table: unshadowed, no draw
    const bool rig = uses_rig(W);
    V3 sum = rig ? rig_fill(W, s) : v3(0.0f);
    for (uint32_t k = 0; k < 4u; k++) {
        Shadowed q = unshadowed();
        if (k == 0u) {
            if (rig) q = rig_query(W, 0u, s, seed);
            else q = lamp_query(W, s, seed);
        } else if (k == 1u) {
            if (rig) q = rig_query(W, 1u, s, seed);
        } else if (k == 2u) {
            q = glow_query(W, s, seed);
        }
        if (maxc(q.c) > 0.0f) sum += q.c * visible(W, s.pos, q.dir, q.dist);
    }
    return sum;
}

V3 indirect(World& W, V3 pos, V3 n, uint32_t* seed, bool bounce) {
    const V3 env = v3(W.p->env[0], W.p->env[1], W.p->env[2]);
    const bool lit = W.p->envmap != 0u || dot(env, env) > 0.0f;
    const uint32_t glow = (uint32_t)W.S->lamp_face.size();
    if (glow == 0u && !lit) {
        const V3 dir = cosine_dir(n, seed);
        // env_at(dir) * mix(0.25, 1, visible(...)): exactly zero for a black
        // world, so the occlusion ray is traced only when it can matter.
        if (env.x == 0.0f && env.y == 0.0f && env.z == 0.0f) return v3(0.0f);
        return env_at(W, dir) * mixf(0.25f, 1.0f, visible(W, pos, dir, W.ao));
    }
    const bool sampled = W.p->env_cdf != 0u;
    const uint32_t depth = bounce ? (W.p->bounces != 0u ? W.p->bounces : (sampled ? 4u : 1u)) : 1u;
    V3 acc = v3(0.0f), thr = v3(1.0f), org = pos, nrm = n;
    bool escaped = false;
    float min_pdf = 3.0e38f;
    bool through = false;
    V3 dir = v3(0.0f, 0.0f, 1.0f);
    float pb = 1.0f;
    for (uint32_t b = 0; b < depth; b++) {
        if (!through) {
            dir = cosine_dir(nrm, seed);
            pb = fmaxw(dot(nrm, dir), 0.0f) / PI;
        }
        through = false;
        min_pdf = fminw(min_pdf, pb);
        const Hit h = trace(W, org, dir, INF, false);
        if (h.tri == NONE) {
            acc += thr * env_at(W, dir) * 1.0f;
            escaped = true;
            break;
        }
        if (!bounce) break;
        const Tri t = tri_of(W, h.tri, h.inst);
        const V3 ng0 = normalize(cross(t.b - t.a, t.c - t.a));
        const V3 ng = dot(ng0, dir) < 0.0f ? ng0 : -ng0;
        const V3 hit = org + dir * h.t + ng * (W.eps + h.t * 1e-5f);
        const V3 base = vmax(v3(t.color[0], t.color[1], t.color[2]), v3(0.0f));
        const float rough = fmaxw(t.rough, glossy_floor(min_pdf));
        const bool glossy = true;  // caustic_reflective with integrator.x 0
        const V3 fd = glossy ? dielectric_f0(t.ior) : v3(0.0f);
        const float metal = glossy ? t.metal : 0.0f;
        const float tw = t.trans * (1.0f - t.metal);
        V3 albedo = base * (1.0f - t.metal) * (1.0f - tw);
        if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxw(dot(ng, -dir), 1e-4f));
        acc += thr * glow_mis(W, t, h, nrm, dir);
        const float near = (!lit && h.t <= W.ao) ? 0.25f : 1.0f;
        const Surf s = plain_surf(hit, ng, -dir, albedo, vmix(fd, base, metal), rough);
        acc += thr * direct(W, s, seed, true) * near;
        if (tw > 0.0f && rnd(seed) < tw) {
            thr *= v3(std::sqrt(base.x), std::sqrt(base.y), std::sqrt(base.z));
            const V3 at = org + dir * h.t;
            org = at - ng * through_lift(W, at, h.t);
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
    (void)escaped;  // the tail needs an environment image
    return acc;
}

V3 bounce_light(World& W, const Hit& h, V3 org, V3 d, float min_pdf, uint32_t* seed) {
    const Tri t = tri_of(W, h.tri, h.inst);
    const V3 ng0 = normalize(cross(t.b - t.a, t.c - t.a));
    const V3 ng = dot(ng0, d) < 0.0f ? ng0 : -ng0;
    const V3 pos = org + d * h.t + ng * (W.eps + h.t * 1e-5f);
    const V3 base = vmax(v3(t.color[0], t.color[1], t.color[2]), v3(0.0f));
    const float rough = fmaxw(t.rough, glossy_floor(min_pdf));
    const V3 fd = dielectric_f0(t.ior);
    V3 albedo = base * (1.0f - t.metal);
    if (maxc(albedo) > 0.0f) albedo *= under_layer(fd, rough, fmaxw(dot(ng, -d), 1e-4f));
    const Surf s = plain_surf(pos, ng, -d, albedo, vmix(fd, base, t.metal), rough);
    return direct(W, s, seed, false) + s.albedo * env_at(W, ng) * 0.8f + t.emit;
}

V3 clamp_light(V3 l, float limit) {
    const float m = maxc(l);
    if (limit <= 0.0f || m <= limit) return l;
    return l * (limit / m);
}

// ---- util.wgsl guide / emit ----

void guide(World& W, uint32_t i, V3 albedo, V3 n, float dist) {
    uint32_t* px = W.px;
    const uint32_t N = W.n;
    const uint32_t a = 7 * N + 3 * i, b = 10 * N + 3 * i, c = 13 * N + i;
    const bool keep = W.frame > 0u;
    const V3 old_a = keep ? v3(f_of(px[a]), f_of(px[a + 1]), f_of(px[a + 2])) : v3(0.0f);
    const V3 old_n = keep ? v3(f_of(px[b]), f_of(px[b + 1]), f_of(px[b + 2])) : v3(0.0f);
    const float old_d = keep ? f_of(px[c]) : 0.0f;
    const V3 sa = old_a + albedo;
    const V3 sn = old_n + n;
    px[a] = u_of(sa.x);
    px[a + 1] = u_of(sa.y);
    px[a + 2] = u_of(sa.z);
    px[b] = u_of(sn.x);
    px[b + 1] = u_of(sn.y);
    px[b + 2] = u_of(sn.z);
    px[c] = u_of(old_d + dist);
}

void emit(World& W, uint32_t i, V3 lin, V3 over_rgb, float over_a, float cover, float missed) {
    uint32_t* px = W.px;
    const uint32_t N = W.n;
    const uint32_t a = N + 3 * i, g = 20 * N + 3 * i, gc = 23 * N + i, fc = 24 * N + i, mc = 33 * N + i;
    const bool keep = W.frame > 0u;
    const float gone = (keep ? f_of(px[mc]) : 0.0f) + missed;
    px[mc] = u_of(gone);
    const uint32_t cn = 31 * N + i;
    const uint32_t taken = (keep ? px[cn] : 0u) + 1u;
    px[cn] = taken;
    const float k = (float)taken;
    const float film = (keep ? f_of(px[fc]) : 0.0f) + cover;
    px[fc] = u_of(film);
    const V3 l = (keep ? v3(f_of(px[a]), f_of(px[a + 1]), f_of(px[a + 2])) : v3(0.0f)) + lin;
    const V3 gs = (keep ? v3(f_of(px[g]), f_of(px[g + 1]), f_of(px[g + 2])) : v3(0.0f)) + over_rgb;
    const float cov = (keep ? f_of(px[gc]) : 0.0f) + over_a;
    px[a] = u_of(l.x);
    px[a + 1] = u_of(l.y);
    px[a + 2] = u_of(l.z);
    px[g] = u_of(gs.x);
    px[g + 1] = u_of(gs.y);
    px[g + 2] = u_of(gs.z);
    px[gc] = u_of(cov);
    // util.wgsl:126-132: Adaptive Sampling's half image takes the odd
    // samples at double weight.
    if (W.p->adapt[3] != 0.0f && (W.frame & 1u)) {
        const uint32_t x = 26 * N + 3 * i;
        const V3 half = (keep ? v3(f_of(px[x]), f_of(px[x + 1]), f_of(px[x + 2])) : v3(0.0f)) + lin * 2.0f;
        px[x] = u_of(half.x);
        px[x + 1] = u_of(half.y);
        px[x + 2] = u_of(half.z);
    }
    const V3 shown = view_transform_of(l / fmaxw(k - gone, 1.0f), W.p->view) * (1.0f - cov / k) + gs / k;
    const uint32_t b = 4 * N + 3 * i;
    px[b] = u_of(shown.x);
    px[b + 1] = u_of(shown.y);
    px[b + 2] = u_of(shown.z);
    px[i] = pack(shown, film / k);
}

float srgb_to_linear1(float c) { return c <= 0.04045f ? c / 12.92f : pm_pow((c + 0.055f) / 1.055f, 2.4f); }

// ---- util.wgsl:185-272 the floor grid overlay ----

struct Over {
    V3 c;
    float a;
};

// floor_over: the floor's lines and its X and Y axes, premultiplied.
Over floor_over(const phx_camera* p, V3 o, V3 d, float t_hit, float px_) {
    if (p->grid <= 0.0f || std::fabs(d.z) < 1e-6f) return Over{v3(0.0f), 0.0f};
    const float t = -o.z / d.z;
    if (t <= 0.0f || t >= t_hit) return Over{v3(0.0f), 0.0f};
    const V3 q = o + d * t;
    float foot = px_;
    if (p->persp != 0u) foot = px_ * t * p->units / p->dist;
    const float want = foot * 24.0f;
    const float lg = pm_log2(fmaxw(want, 1e-9f)) / pm_log2(10.0f);
    const float lvl = std::floor(lg);
    const float f = lg - lvl;
    const float g0 = pm_pow(10.0f, lvl);
    const float g1 = g0 * 10.0f;
    const float half_w = foot * 0.5f;
    const float aa = foot;
    const float c0x = q.x / g0, c0y = q.y / g0;
    const float c1x = q.x / g1, c1y = q.y / g1;
    // WGSL round: to nearest, ties to even
    const float d0x = std::fabs(c0x - std::nearbyint(c0x)) * g0, d0y = std::fabs(c0y - std::nearbyint(c0y)) * g0;
    const float d1x = std::fabs(c1x - std::nearbyint(c1x)) * g1, d1y = std::fabs(c1y - std::nearbyint(c1y)) * g1;
    const float l0 = fmaxw(1.0f - smoothstep(half_w, half_w + aa, d0x), 1.0f - smoothstep(half_w, half_w + aa, d0y));
    const float l1 = fmaxw(1.0f - smoothstep(half_w, half_w + aa, d1x), 1.0f - smoothstep(half_w, half_w + aa, d1y));
    const float fine = (1.0f - f) * (1.0f - f);
    const float line = fmaxw(l0 * fine * 0.6f, l1);
    const float horizon = clampf(std::fabs(d.z) * 4.0f, 0.0f, 1.0f);
    float depth = 1.0f;
    if (p->persp != 0u) {
        const float r = t * p->units / (p->dist * 6.0f);
        depth = 1.0f / (1.0f + r * r);
    }
    const float fade = horizon * depth;
    const float w0 = line * p->grid_color[3] * fade * ((p->grid_hide & 1u) != 0u ? 0.0f : 1.0f);
    V3 c = v3(p->grid_color[0], p->grid_color[1], p->grid_color[2]) * w0;
    float a = w0;
    const float ax = 1.0f - smoothstep(half_w, half_w + aa, std::fabs(q.y));
    const float ay = 1.0f - smoothstep(half_w, half_w + aa, std::fabs(q.x));
    const float w1 = ax * 0.85f * fade * ((p->grid_hide & 2u) != 0u ? 0.0f : 1.0f);
    c = c * (1.0f - w1) + v3(0.85f, 0.3f, 0.33f) * w1;
    a = a * (1.0f - w1) + w1;
    const float w2 = ay * 0.85f * fade * ((p->grid_hide & 4u) != 0u ? 0.0f : 1.0f);
    c = c * (1.0f - w2) + v3(0.47f, 0.72f, 0.2f) * w2;
    a = a * (1.0f - w2) + w2;
    return Over{c, a};
}

// z_axis_over: the vertical line through the origin.
Over z_axis_over(const phx_camera* p, V3 o, V3 d, float t_hit, float px_) {
    const float a = d.x * d.x + d.y * d.y;
    if (a < 1e-12f) return Over{v3(0.0f), 0.0f};
    const float t = -(o.x * d.x + o.y * d.y) / a;
    if (t <= 0.0f || t >= t_hit) return Over{v3(0.0f), 0.0f};
    float foot = px_;
    if (p->persp != 0u) foot = px_ * t * p->units / p->dist;
    const V3 at = o + d * t;
    const float r = std::sqrt(at.x * at.x + at.y * at.y);
    const float w = (1.0f - smoothstep(foot * 0.5f, foot * 1.5f, r)) * 0.85f;
    return Over{v3(0.25f, 0.53f, 0.92f) * w, w};
}

// grid_over: the floor, then the Z axis laid over it when asked for.
Over grid_over(const phx_camera* p, V3 o, V3 d, float t_hit, float px_) {
    Over g = floor_over(p, o, d, t_hit, px_);
    if (p->grid > 0.0f && (p->grid_hide & 8u) != 0u) {
        const Over z = z_axis_over(p, o, d, t_hit, px_);
        g = Over{g.c * (1.0f - z.a) + z.c, g.a * (1.0f - z.a) + z.a};
    }
    return g;
}

struct CamRay {
    V3 o, d;
};

// shade.wgsl:66-95 (pinhole or orthographic, phiray's own pixel filter).
CamRay camera_ray(const World& W, uint32_t i, uint32_t* seed) {
    const phx_camera* p = W.p;
    const float fw = (float)p->w, fh = (float)p->h;
    const float su = ((float)(i % p->w) + 0.5f) / fw - 0.5f;
    const float sv = ((float)(i / p->w) + 0.5f) / fh - 0.5f;
    const float u = rnd(seed);
    const float v = rnd(seed);
    const float jox = u - 0.5f, joy = v - 0.5f;
    const float jx = jox / fw;
    const float jy = joy / fh;
    const float vx = (su + jx - p->pan[0]) / p->scale;
    const float vy = -((sv + jy) / p->aspect - p->pan[1]) / p->scale;
    CamRay r;
    if (p->persp != 0u) {
        r.o = vec(p->pivot) + vec(p->back) * (p->dist / p->units);
        r.d = normalize(vec(p->right) * vx + vec(p->up) * vy - vec(p->back) * p->dist);
    } else {
        r.o = vec(p->pivot) + (vec(p->right) * vx + vec(p->up) * vy + vec(p->back) * 1.0e4f) / p->units;
        r.d = -vec(p->back);
    }
    return r;
}

// shade.wgsl main for pixel i, frame W.frame.
void shade_main(World& W, uint32_t i) {
    const phx_camera* p = W.p;
    uint32_t* px = W.px;
    const uint32_t N = W.n;
    if (W.frame == 0u) {
        px[29 * N + i] = 0u;
        px[30 * N + i] = 0u;
    }
    // shade.wgsl:44-64: past frame 0 only the open pixels are traced (the
    // list gather.wgsl built from the settled flags of the last tail).
    if (p->adapt[3] != 0.0f && px[30 * N + i] != 0u) return;
    uint32_t seed = hash(i * 9781u + W.frame * 6271u + 1u);
    const CamRay cr = camera_ray(W, i, &seed);
    V3 o = cr.o, d = cr.d;
    // shade.wgsl:96-103: a pixel's footprint for the grid, the first ray and
    // the first surface's distance
    const float pix = 1.0f / (p->scale * p->units * (float)p->w);
    const V3 o0 = o, d0 = d;
    float first_t = INF;
    const float across = (float)(i % p->w) / fmaxw((float)p->w * 0.5f, 1.0f);
    const V3 sky = v3(p->sky[0], p->sky[1], p->sky[2]) + v3(p->sky[3]) * (1.0f - clampf(across, 0.0f, 1.0f));
    px[25 * N + i] = 0u;  // outline_store(i, 0)
    V3 col = v3(0.0f), thr = v3(1.0f);
    const uint32_t see_through = 8u, through = 8u;
    const bool glossy_on = true, diffuse_on = true;
    uint32_t n_see = 0, n_through = 0;
    const uint32_t passes = see_through + through + 1u;
    for (uint32_t bounce = 0; bounce < passes; bounce++) {
        const Hit h = trace(W, o, d, INF, false);
        if (h.tri == NONE) {
            if (bounce == 0u) {
                const Over g = grid_over(p, o, d, INF, pix);
                guide(W, i, v3(srgb_to_linear1(sky.x), srgb_to_linear1(sky.y), srgb_to_linear1(sky.z)), -d, -1.0f);
                emit(W, i, v3(0.0f), sky * (1.0f - g.a) + g.c, 1.0f, 1.0f, 1.0f);
                return;
            }
            col += thr * env_at(W, d);
            break;
        }
        if (bounce == 0u) {
            first_t = h.t;
            px[25 * N + i] = h.inst + 1u;
        }
        const Tri t = tri_of(W, h.tri, h.inst);
        const float w = 1.0f - h.u - h.v;
        const V3 hit = o + d * h.t;
        const V3 ng0 = world_ng(t);
        const bool front = dot(ng0, d) < 0.0f;
        const V3 ng = front ? ng0 : -ng0;
        V3 n = t.na * w + t.nb * h.u + t.nc * h.v;
        n = dot(n, n) > 1e-12f ? normalize(n) * (front ? 1.0f : -1.0f) : ng;
        if (dot(n, -d) < 0.0f) n = ng;
        const V3 off = ng * hit_lift(W, h.t);
        const V3 past = ng * through_lift(W, hit, h.t);
        const V3 pos = hit + off;
        const V3 base = vmax(v3(t.color[0], t.color[1], t.color[2]), v3(0.0f));
        const float alpha = t.color[3];
        const float rough = t.rough;
        const float metal = t.metal;
        const V3 emit_c = t.emit;
        if (bounce == 0u) guide(W, i, base, n, h.t);
        if (rnd(&seed) >= alpha) {
            n_see++;
            if (n_see > see_through) break;
            o = hit - past;
            continue;
        }
        col += thr * emit_c;
        const float bleed = scatter_bleed(t.sss, t.sss_radius);
        const V3 fd = dielectric_f0(t.ior);
        V3 diffuse = base * (1.0f - metal);
        if (maxc(diffuse) > 0.0f) diffuse *= under_layer_real(t.ior, fmaxw(rough, 0.04f), fmaxw(dot(n, -d), 1e-4f));
        const Surf s{pos,   n,      -d,     diffuse, vmix(fd, base, metal), fmaxw(rough, 0.04f), bleed,
                     scatter_tint(t.sss_radius), t.sheen, t.sheen_rough, t.sheen_tint, t.coat, t.coat_rough, t.ior,
                     1.0f - metal};
        const float opaque = 1.0f - t.trans * (1.0f - metal);
        V3 c = v3(0.0f);
        if (opaque > 0.0f) c = direct(W, s, &seed, true) * opaque;
        if (opaque < 1.0f) {
            const Surf shine{pos,       n,           -d,    v3(0.0f), s.f0,         s.rough, 0.0f, v3(1.0f),
                             0.0f,      t.sheen_rough, t.sheen_tint, t.coat, t.coat_rough, s.eta, s.dielectric};
            c += direct(W, shine, &seed, true) * (1.0f - opaque);
        }
        c = clamp_light(c, p->limit[0]);
        V3 bounced = v3(0.0f);
        const V3 diffuse_weight = vmix(s.albedo, s.albedo * s.sss_tint, bleed) * opaque;
        const V3 lw = v3(0.2126f, 0.7152f, 0.0722f);
        const float ndv = fmaxw(dot(n, -d), 1e-4f);
        const V3 gloss_guess = s.f0 + (v3(1.0f) - s.f0) * pm_pow(1.0f - ndv, 5.0f);
        const float pd = dot(vmax(diffuse_weight, v3(0.0f)), lw);
        const float pg = glossy_on ? dot(gloss_guess, lw) : 0.0f;
        float p_diffuse = (pd + pg > 0.0f) ? pd / (pd + pg) : 1.0f;
        if (pd > 0.0f && pg > 0.0f) p_diffuse = clampf(p_diffuse, 0.15f, 0.85f);
        const bool take_diffuse = rnd(&seed) < p_diffuse;
        if (take_diffuse && pd > 0.0f) bounced += diffuse_weight * indirect(W, pos, n, &seed, diffuse_on) / p_diffuse;
        const V3 v = -d;
        const V3 tx = normalize(onb(n, 1.0f, 0.0f));
        const V3 ty = cross(n, tx);
        const float ggx_a = s.rough * s.rough;
        const V3 wi_local = v3(dot(v, tx), dot(v, ty), dot(v, n));
        const float ra = rnd(&seed);
        const float rb = rnd(&seed);
        const V3 h_local = ggx_sample_vndf(wi_local, ggx_a, ra, rb);
        const V3 hw = normalize(tx * h_local.x + ty * h_local.y + n * h_local.z);
        const V3 refl = reflect(d, hw);
        const float cos_hi = fmaxw(dot(hw, v), 0.0f);
        const float cos_no = dot(n, refl);
        const V3 fres = fresnel_of(s, cos_hi);
        if (!take_diffuse && glossy_on && dot(refl, ng) > 0.0f && cos_hi > 0.0f && cos_no > 0.0f) {
            const Hit rh = trace(W, pos, refl, INF, false);
            V3 rc = env_at(W, refl);
            const float wg = 1.0f;
            if (rh.tri != NONE) rc = bounce_light(W, rh, pos, refl, ggx_pdf(s, refl), &seed);
            bounced += fres * rc * ggx_weight(ggx_a * ggx_a, fmaxw(dot(n, v), 1e-4f), cos_no) * wg / (1.0f - p_diffuse);
        }
        c += clamp_light(bounced, p->limit[1]);
        col += thr * c;
        const float tw = t.trans * (1.0f - metal);
        if (tw <= 0.0f) break;
        n_through++;
        if (n_through > through) break;
        const float eta = front ? 1.0f / t.ior : t.ior;
        V3 nd = refract(d, n, eta);
        if (dot(nd, nd) < 1e-6f) {
            nd = reflect(d, n);
            o = hit + past;
            thr *= tw;
        } else {
            o = hit - past;
            thr *= tw * v3(std::sqrt(base.x), std::sqrt(base.y), std::sqrt(base.z)) * (v3(1.0f) - fres);
        }
        d = cone_dir(normalize(nd), s.rough * s.rough, &seed);
        if (maxc(thr) < 0.01f) break;
    }
    const Over g = grid_over(p, o0, d0, first_t, pix);
    emit(W, i, col, g.c, g.a, 1.0f, 0.0f);
}

void setup(Shared& S, World& W, const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats,
           const float* normals, uint32_t leaf, bool sah = false) {
    W.S = &S;
    std::vector<orc_aabb> boxes(nfaces);
    for (uint32_t f = 0; f < nfaces; f++) {
        orc_aabb b;
        std::memset(&b, 0, sizeof b);
        const uint32_t* q = faces + 4 * (size_t)f;
        for (int k = 0; k < 3; k++) {
            const float a = verts[4 * (size_t)q[0] + k], bb = verts[4 * (size_t)q[1] + k], c = verts[4 * (size_t)q[2] + k];
            b.lo[k] = fminw(fminw(a, bb), c);
            b.hi[k] = fmaxw(fmaxw(a, bb), c);
        }
        boxes[f] = b;
    }
    S.nodes.assign(2 * (size_t)nfaces - 1, orc_node{});
    S.order.assign(nfaces, 0);
    uint32_t depth = 0;
    if (sah) {
        // the binned SAH tree phiray's tracer builds (forest.rs:49 build_sah)
        S.nodes.resize(orc_build_sah(boxes.data(), nfaces, leaf ? leaf : 4, S.nodes.data(), S.order.data(), &depth));
    } else {
        orc_build(boxes.data(), nfaces, leaf ? leaf : 4, S.nodes.data(), S.order.data(), &depth);
    }
    W.verts = verts;
    W.normals = normals;
    W.faces = faces;
    W.mats = mats;
    // lamp.rs table_of, faces in leaf order, one instance.
    std::vector<float> pw;
    for (uint32_t s = 0; s < nfaces; s++) {
        const uint32_t* q = faces + 4 * (size_t)S.order[s];
        const float* m = mats + 32 * (size_t)q[3];
        const float glow = 0.2126f * m[8] + 0.7152f * m[9] + 0.0722f * m[10];
        if (glow <= 0.0f) continue;
        const V3 a = W.vert(q[0]), b = W.vert(q[1]), c = W.vert(q[2]);
        const float e1[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
        const float e2[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
        const float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        float sq = 0.0f;
        for (int k = 0; k < 3; k++) sq += cr[k] * cr[k];
        const float p = 0.5f * std::sqrt(sq) * glow;
        if (p > 0.0f) {
            S.lamp_face.push_back(s);
            S.lamp_inst.push_back(0u);
            pw.push_back(p);
        }
    }
    float total = 0.0f;
    for (float p : pw) total += p;
    float run = 0.0f;
    for (float p : pw) {
        run += p;
        S.lamp_cdf.push_back(run / total);
    }
    // Forest::extent (forest.rs:192-200) and Tracer::sample_in's ao / eps.
    float e = 0.0f;
    for (int k = 0; k < 3; k++) {
        const float dk = S.nodes[0].hi.p[k] - S.nodes[0].lo.p[k];
        e += dk * dk;
    }
    S.extent = fmaxw(std::sqrt(e), 1e-3f);
}

// Instance::inverse and words (instance.rs): rows of the world matrix and
// of its inverse (the upper 3 x 3 inverted, the translation undone; zero for
// a singular matrix), and the flags.
Inst inst_of(const phx_instance& src) {
    Inst in;
    const float* m = src.world;  // m[col][row] at m[4 * col + row]
    auto a = [&](int r, int c) { return m[4 * c + r]; };
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) in.row[r][c] = m[4 * c + r];
    const float det = a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
                      a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
    if (std::fabs(det) < 1e-20f) {
        std::memset(in.inv, 0, sizeof in.inv);
    } else {
        const float d = 1.0f / det;
        const float inv[3][3] = {
            {(a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * d, (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * d,
             (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * d},
            {(a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * d, (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * d,
             (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * d},
            {(a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * d, (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * d,
             (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * d},
        };
        const float t[3] = {m[12], m[13], m[14]};
        for (int r = 0; r < 3; r++) {
            for (int c = 0; c < 3; c++) in.inv[r][c] = inv[r][c];
            in.inv[r][3] = -((inv[r][0] * t[0] + inv[r][1] * t[1]) + inv[r][2] * t[2]);
        }
    }
    bool identity = true;
    for (int k = 0; k < 16; k++) identity = identity && m[k] == ((k % 5 == 0) ? 1.0f : 0.0f);
    in.mesh = src.mesh;
    in.flags = (identity ? 1u : 0u) | (src.casts_shadow ? 0u : 2u) | (det < 0.0f ? 4u : 0u);
    return in;
}

// Forest::retlas (forest.rs:107-121) with the LBVH: the top tree over the
// world boxes (Instance::world_box of each mesh's root bounds) of the
// instances whose mesh has faces, one instance a leaf; then the extent.
void retlas(Shared& S) {
    std::vector<uint32_t> placed;
    std::vector<orc_aabb> boxes;
    for (uint32_t i = 0; i < S.insts.size(); i++) {
        const Inst& in = S.insts[i];
        if (in.mesh >= S.meshes.size() || S.meshes[in.mesh].nodes.empty()) continue;
        const orc_node& root = S.meshes[in.mesh].nodes[0];
        orc_aabb b;
        std::memset(&b, 0, sizeof b);
        for (int k = 0; k < 3; k++) {  // Aabb::default(): [f32::MAX; 3], [f32::MIN; 3]
            b.lo[k] = 3.40282347e38f;
            b.hi[k] = -3.40282347e38f;
        }
        for (int k = 0; k < 8; k++) {
            const float c[3] = {(k & 1) == 0 ? root.lo.p[0] : root.hi.p[0], (k & 2) == 0 ? root.lo.p[1] : root.hi.p[1],
                                (k & 4) == 0 ? root.lo.p[2] : root.hi.p[2]};
            for (int r = 0; r < 3; r++) {
                const float w = ((in.row[r][0] * c[0] + in.row[r][1] * c[1]) + in.row[r][2] * c[2]) + in.row[r][3];
                b.lo[r] = fminw(b.lo[r], w);
                b.hi[r] = fmaxw(b.hi[r], w);
            }
        }
        placed.push_back(i);
        boxes.push_back(b);
    }
    const uint32_t n = (uint32_t)placed.size();
    S.nodes.assign(n ? 2 * (size_t)n - 1 : 0, orc_node{});
    std::vector<uint32_t> order(n);
    uint32_t depth = 0;
    if (n) orc_build(boxes.data(), n, 1, S.nodes.data(), order.data(), &depth);
    S.inst_order.resize(n);
    for (uint32_t s = 0; s < n; s++) S.inst_order[s] = placed[order[s]];
    float e = 0.0f;
    if (n) {
        for (int k = 0; k < 3; k++) {
            const float dk = S.nodes[0].hi.p[k] - S.nodes[0].lo.p[k];
            e += dk * dk;
        }
    }
    S.extent = fmaxw(std::sqrt(e), 1e-3f);
}

// lamp.rs table_of with instances: every emissive slot (slot order), once
// for each instance of its mesh (instance order), by its world area times
// its emitted luminance.
void relight(Shared& S, const World& W) {
    S.lamp_face.clear();
    S.lamp_inst.clear();
    S.lamp_cdf.clear();
    std::vector<std::vector<uint32_t>> by_mesh(S.meshes.size());
    for (uint32_t i = 0; i < S.insts.size(); i++)
        if (S.insts[i].mesh < S.meshes.size()) by_mesh[S.insts[i].mesh].push_back(i);
    std::vector<float> pw;
    for (uint32_t k = 0; k < S.meshes.size(); k++) {
        for (uint32_t s = S.meshes[k].lo; s < S.meshes[k].hi; s++) {
            const uint32_t* q = W.faces + 4 * (size_t)S.order[s];
            const float* m = W.mats + 32 * (size_t)q[3];
            const float glow = 0.2126f * m[8] + 0.7152f * m[9] + 0.0722f * m[10];
            if (glow <= 0.0f) continue;
            for (uint32_t i : by_mesh[k]) {
                const Inst& in = S.insts[i];
                auto corner = [&](uint32_t v) {
                    const float* p = W.verts + 4 * (size_t)v;
                    auto r = [&](const float* row) { return ((row[0] * p[0] + row[1] * p[1]) + row[2] * p[2]) + row[3]; };
                    return v3(r(in.row[0]), r(in.row[1]), r(in.row[2]));
                };
                const V3 a = corner(q[0]), b = corner(q[1]), c = corner(q[2]);
                const float e1[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
                const float e2[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
                const float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                     e1[0] * e2[1] - e1[1] * e2[0]};
                float sq = 0.0f;
                for (int j = 0; j < 3; j++) sq += cr[j] * cr[j];
                const float p = 0.5f * std::sqrt(sq) * glow;
                if (p > 0.0f) {
                    S.lamp_face.push_back(s);
                    S.lamp_inst.push_back(i);
                    pw.push_back(p);
                }
            }
        }
    }
    float total = 0.0f;
    for (float p : pw) total += p;
    float run = 0.0f;
    for (float p : pw) {
        run += p;
        S.lamp_cdf.push_back(run / total);
    }
}

// Forest::build (forest.rs:44-61) with each mesh's LBVH: the meshes' trees
// in their own space, the slot order (each mesh's faces permuted within its
// range), the instances, the top tree and the emitter table.
void setup_instanced(Shared& S, World& W, const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats,
                     const float* normals, uint32_t leaf, const phx_mesh* meshes, uint32_t nmeshes,
                     const phx_instance* insts, uint32_t ninsts) {
    W.S = &S;
    W.verts = verts;
    W.normals = normals;
    W.faces = faces;
    W.mats = mats;
    S.leaf = leaf ? leaf : 4;
    S.order.resize(nfaces);
    for (uint32_t f = 0; f < nfaces; f++) S.order[f] = f;
    S.meshes.assign(nmeshes, MeshTree{});
    for (uint32_t k = 0; k < nmeshes; k++) {
        MeshTree& mt = S.meshes[k];
        mt.lo = meshes[k].face_lo;
        mt.hi = meshes[k].face_hi;
        const uint32_t n = mt.hi - mt.lo;
        if (n == 0) continue;
        std::vector<orc_aabb> boxes(n);
        for (uint32_t f = 0; f < n; f++) {
            orc_aabb b;
            std::memset(&b, 0, sizeof b);
            const uint32_t* q = faces + 4 * (size_t)(mt.lo + f);
            for (int j = 0; j < 3; j++) {
                const float a = verts[4 * (size_t)q[0] + j], bb = verts[4 * (size_t)q[1] + j], c = verts[4 * (size_t)q[2] + j];
                b.lo[j] = fminw(fminw(a, bb), c);
                b.hi[j] = fmaxw(fmaxw(a, bb), c);
            }
            boxes[f] = b;
        }
        mt.nodes.assign(2 * (size_t)n - 1, orc_node{});
        std::vector<uint32_t> order(n);
        uint32_t depth = 0;
        orc_build(boxes.data(), n, S.leaf, mt.nodes.data(), order.data(), &depth);
        for (uint32_t sl = 0; sl < n; sl++) S.order[mt.lo + sl] = mt.lo + order[sl];
    }
    S.insts.resize(ninsts);
    for (uint32_t i = 0; i < ninsts; i++) S.insts[i] = inst_of(insts[i]);
    retlas(S);
    relight(S, W);
}

}  // namespace

extern "C" {

struct OrcScene {
    Shared S;
    World W0;
};

void* orc_scene_new(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, const float* normals,
                    uint32_t leaf) {
    auto* h = new OrcScene();
    setup(h->S, h->W0, verts, faces, nfaces, mats, normals, leaf);
    return h;
}

void* orc_scene_new_sah(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats,
                        const float* normals, uint32_t leaf) {
    auto* h = new OrcScene();
    setup(h->S, h->W0, verts, faces, nfaces, mats, normals, leaf, true);
    return h;
}

void orc_scene_free(void* handle) { delete (OrcScene*)handle; }

void* orc_scene_new_instanced(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats,
                              const float* normals, uint32_t leaf, const phx_mesh* meshes, uint32_t nmeshes,
                              const phx_instance* insts, uint32_t ninsts) {
    auto* h = new OrcScene();
    setup_instanced(h->S, h->W0, verts, faces, nfaces, mats, normals, leaf, meshes, nmeshes, insts, ninsts);
    return h;
}

// Tracer::reinstance (pose.rs:105-120): new matrices for the same instances,
// the top tree again, the emitter table again.
void orc_scene_reinstance(void* handle, const phx_instance* insts, uint32_t ninsts) {
    OrcScene* h = (OrcScene*)handle;
    for (uint32_t i = 0; i < ninsts && i < h->S.insts.size(); i++) {
        const uint32_t mesh = h->S.insts[i].mesh;
        h->S.insts[i] = inst_of(insts[i]);
        h->S.insts[i].mesh = mesh;
    }
    retlas(h->S);
    relight(h->S, h->W0);
}

// Primary hits and ray-buffer walks of a scene handle (as orc_primary and
// orc_trace_rays, which build a single-instance scene of their own).
void orc_scene_primary(void* handle, const phx_camera* cam, uint32_t frame, uint32_t* ids, float* ts, uint32_t* insts) {
    const OrcScene* h = (const OrcScene*)handle;
    const uint32_t n = cam->w * cam->h;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        World W = h->W0;
        W.p = cam;
        W.n = n;
        uint32_t seed = hash((uint32_t)i * 9781u + frame * 6271u + 1u);
        const CamRay cr = camera_ray(W, (uint32_t)i, &seed);
        const Hit hh = trace(W, cr.o, cr.d, INF, false);
        ids[i] = hh.tri == NONE ? NONE : h->S.order[hh.tri];
        ts[i] = hh.t;
        if (insts) insts[i] = hh.tri == NONE ? NONE : hh.inst;
    }
}

void orc_scene_trace_rays(void* handle, const float* rays, uint32_t n, float* hits, int any_hit) {
    const OrcScene* h = (const OrcScene*)handle;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        World W = h->W0;
        const float* r = rays + 8 * (size_t)i;
        const Hit hh = trace(W, v3(r[0], r[1], r[2]), v3(r[4], r[5], r[6]), r[3], any_hit != 0);
        hits[4 * i] = hh.t;
        hits[4 * i + 1] = f_of(hh.tri == NONE ? NONE : h->S.order[hh.tri]);
        hits[4 * i + 2] = hh.u;
        hits[4 * i + 3] = hh.v;
    }
}

// adapt.wgsl and gather.wgsl: the tail after `sample` — the convergence
// check at a step boundary past the minimum, the dilation over the four
// neighbours, and the open-pixel list (pixel order) with its length at 34n.
static void adapt_tail(const phx_camera* cam, uint32_t* px, uint32_t sample) {
    const uint32_t w = cam->w, h = cam->h, n = w * h;
    const uint32_t min_samples = cam->adapt[1] > 0.0f ? (uint32_t)cam->adapt[1] : 0u;
    const uint32_t step = cam->adapt[2] >= 1.0f ? (uint32_t)cam->adapt[2] : 1u;
    if (sample > min_samples && (sample & (step - 1u)) == step - 1u) {
        for (uint32_t i = 0; i < n; i++) {
            if (px[29 * n + i] != 0u) continue;
            const uint32_t a = n + 3 * i, x = 26 * n + 3 * i;
            const float fr = f_of(px[a]), fg = f_of(px[a + 1]), fb = f_of(px[a + 2]);
            const float hr = f_of(px[x]), hg = f_of(px[x + 1]), hb = f_of(px[x + 2]);
            const uint32_t taken = px[31 * n + i] > 1u ? px[31 * n + i] : 1u;
            const float scale = 1.0f / (float)taken;
            const float error_difference = (std::fabs(fr - hr) + std::fabs(fg - hg) + std::fabs(fb - hb)) * scale;
            const float intensity = (fr + fg + fb) * scale;
            const float error_normalize = intensity < 1.0f ? std::sqrt(intensity) : intensity;
            const float error = error_difference / (0.0001f + error_normalize);
            if (error < cam->adapt[0]) px[29 * n + i] = 1u;
        }
    }
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t x = i % w, y = i / w;
        const uint32_t* f = px + 29 * (size_t)n;
        uint32_t all = f[i];
        if (x > 0u) all = std::min(all, f[i - 1]);
        if (x + 1u < w) all = std::min(all, f[i + 1]);
        if (y > 0u) all = std::min(all, f[i - w]);
        if (y + 1u < h) all = std::min(all, f[i + w]);
        px[30 * (size_t)n + i] = all;
    }
    uint32_t open = 0;
    for (uint32_t i = 0; i < n; i++)
        if (px[30 * (size_t)n + i] == 0u) px[32 * (size_t)n + open++] = i;
    px[34 * (size_t)n] = open;
}

static void scene_trace(void* handle, const phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                        uint64_t* rays_out, uint32_t row0, uint32_t rows, uint64_t* walk);

void orc_scene_trace(void* handle, const phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                     uint64_t* rays_out, uint32_t row0, uint32_t rows) {
    scene_trace(handle, cam, first, spp, px, rays_out, row0, rows, nullptr);
}

// The same, also counting the walks' inner-node visits and triangle tests
// (walk[0], walk[1]): a tree's cost on a real ray load.
void orc_scene_trace_walk(void* handle, const phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                          uint64_t* rays_out, uint32_t row0, uint32_t rows, uint64_t* walk) {
    scene_trace(handle, cam, first, spp, px, rays_out, row0, rows, walk);
}

static void scene_trace(void* handle, const phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px,
                        uint64_t* rays_out, uint32_t row0, uint32_t rows, uint64_t* walk) {
    const OrcScene* h = (const OrcScene*)handle;
    uint64_t steps_sum = 0, tests_sum = 0;
    if (cam->adapt[3] != 0.0f) {
        // Adaptive Sampling couples neighbouring pixels between samples:
        // whole frames, sample by sample, each followed by its tail.
        const Shared& S = h->S;
        const uint32_t n = cam->w * cam->h;
        uint64_t total = 0;
        for (uint32_t f = first; f < first + spp; f++) {
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total, steps_sum, tests_sum)
            for (int64_t i = 0; i < (int64_t)n; i++) {
                World W = h->W0;
                W.p = cam;
                W.n = n;
                W.px = px;
                W.ao = cam->ao > 0.0f ? cam->ao : S.extent * 0.08f;
                W.eps = S.extent * 1e-5f;
                W.rays = 0;
                W.frame = f;
                shade_main(W, (uint32_t)i);
                total += W.rays;
                steps_sum += W.steps;
                tests_sum += W.tests;
            }
            adapt_tail(cam, px, f);
        }
        if (rays_out) *rays_out = total;
        if (walk) {
            walk[0] = steps_sum;
            walk[1] = tests_sum;
        }
        return;
    }
    const Shared& S = h->S;
    const uint32_t w = cam->w, hh = cam->h;
    const uint32_t n = w * hh;
    const float ao = cam->ao > 0.0f ? cam->ao : S.extent * 0.08f;
    const float eps = S.extent * 1e-5f;
    const uint32_t r1 = rows ? (row0 + rows < hh ? row0 + rows : hh) : hh;
    uint64_t total = 0;
    // Pixels are independent: threads take runs of 32 pixels, so a band of
    // one row keeps every thread busy too.
#pragma omp parallel reduction(+ : total, steps_sum, tests_sum)
    {
        World W = h->W0;  // the scene is shared; counters are per thread
        W.p = cam;
        W.n = n;
        W.px = px;
        W.ao = ao;
        W.eps = eps;
        W.rays = 0;
#pragma omp for schedule(dynamic, 32)
        for (int64_t i = (int64_t)row0 * w; i < (int64_t)r1 * w; i++) {
            for (uint32_t f = first; f < first + spp; f++) {
                W.frame = f;
                shade_main(W, (uint32_t)i);
            }
        }
        total += W.rays;
        steps_sum += W.steps;
        tests_sum += W.tests;
    }
    if (rays_out) *rays_out = total;
    if (walk) {
        walk[0] = steps_sum;
        walk[1] = tests_sum;
    }
}

void orc_trace(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, const float* normals,
               uint32_t leaf, const phx_camera* cam, uint32_t first, uint32_t spp, uint32_t* px, uint64_t* rays_out,
               uint32_t row0, uint32_t rows) {
    void* h = orc_scene_new(verts, faces, nfaces, mats, normals, leaf);
    orc_scene_trace(h, cam, first, spp, px, rays_out, row0, rows);
    orc_scene_free(h);
}

// show.wgsl: emit's display tail over the sums already in px.
void orc_show(const phx_camera* cam, uint32_t* px) {
    const uint32_t n = cam->w * cam->h;
    for (uint32_t i = 0; i < n; i++) {
        const float k = (float)(px[31 * n + i] > 1u ? px[31 * n + i] : 1u);
        const uint32_t a = n + 3 * i, g = 20 * n + 3 * i;
        const V3 l = v3(f_of(px[a]), f_of(px[a + 1]), f_of(px[a + 2]));
        const V3 gs = v3(f_of(px[g]), f_of(px[g + 1]), f_of(px[g + 2]));
        const float cov = f_of(px[23 * n + i]), film = f_of(px[24 * n + i]), gone = f_of(px[33 * n + i]);
        const V3 shown = view_transform_of(l / fmaxw(k - gone, 1.0f), cam->view) * (1.0f - cov / k) + gs / k;
        const uint32_t b = 4 * n + 3 * i;
        px[b] = u_of(shown.x);
        px[b + 1] = u_of(shown.y);
        px[b + 2] = u_of(shown.z);
        px[i] = pack(shown, film / k);
    }
}

void orc_primary(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, uint32_t leaf,
                 const phx_camera* cam, uint32_t frame, uint32_t* ids, float* ts) {
    Shared S;
    World W0;
    setup(S, W0, verts, faces, nfaces, mats, nullptr, leaf);
    const uint32_t n = cam->w * cam->h;
    W0.ao = cam->ao > 0.0f ? cam->ao : S.extent * 0.08f;
    W0.eps = S.extent * 1e-5f;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        World W = W0;
        W.p = cam;
        W.n = n;
        uint32_t seed = hash((uint32_t)i * 9781u + frame * 6271u + 1u);
        const CamRay cr = camera_ray(W, (uint32_t)i, &seed);
        const Hit h = trace(W, cr.o, cr.d, INF, false);
        ids[i] = h.tri == NONE ? NONE : W.S->order[h.tri];
        ts[i] = h.t;
    }
}

void orc_trace_rays(const float* verts, const uint32_t* faces, uint32_t nfaces, const float* mats, uint32_t leaf,
                    const float* rays, uint32_t n, float* hits, int any_hit) {
    Shared S;
    World W0;
    setup(S, W0, verts, faces, nfaces, mats, nullptr, leaf);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        World W = W0;
        const float* r = rays + 8 * (size_t)i;
        const Hit h = trace(W, v3(r[0], r[1], r[2]), v3(r[4], r[5], r[6]), r[3], any_hit != 0);
        hits[4 * i] = h.t;
        hits[4 * i + 1] = f_of(h.tri == NONE ? NONE : S.order[h.tri]);
        hits[4 * i + 2] = h.u;
        hits[4 * i + 3] = h.v;
    }
}

// The watertight ray/triangle test alone (tri.rs:51-114, bvh.wgsl
// ray_space + tri_t): 1 and (t, u, v) on a hit, 0 otherwise.
int orc_tri_hit(const float* a, const float* b, const float* c, const float* o, const float* d, float* out) {
    float h[3];
    tri_t(v3(a[0], a[1], a[2]), v3(b[0], b[1], b[2]), v3(c[0], c[1], c[2]), v3(o[0], o[1], o[2]),
          ray_space(v3(d[0], d[1], d[2])), h);
    out[0] = h[0];
    out[1] = h[1];
    out[2] = h[2];
    return h[0] < INF ? 1 : 0;
}

// The shared transcendental functions (phiray_math.h) on the host, for
// their accuracy tests: fn 0 exp2, 1 log2, 2 sin, 3 cos, 4 pow(x, y), 5 exp.
void orc_math(int fn, const float* x, const float* y, float* out, uint32_t n) {
    for (uint32_t i = 0; i < n; i++) {
        switch (fn) {
            case 0: out[i] = pm_exp2(x[i]); break;
            case 1: out[i] = pm_log2(x[i]); break;
            case 2: out[i] = pm_sin(x[i]); break;
            case 3: out[i] = pm_cos(x[i]); break;
            case 4: out[i] = pm_pow(x[i], y[i]); break;
            default: out[i] = pm_exp(x[i]); break;
        }
    }
}

}  // extern "C"
