// Oracle (test infrastructure only): C entry points for the Python tests, the smoke
// check and the bench's CPU-baseline leg. Nothing in the product calls these.
#include "orender.h"
#include <cstring>
#include <thread>

using namespace orc;

namespace {
struct OracleScene {
    std::shared_ptr<Scene> scene;
};
void setErr(char* err, int n, const std::string& m) {
    if (err && n > 0) { std::strncpy(err, m.c_str(), n - 1); err[n - 1] = 0; }
}
template <typename F>
void parallelFor(int64_t n, int nthreads, F&& f) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    const int64_t chunk = 256;
    auto work = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            int64_t e = std::min(n, b + chunk);
            for (int64_t i = b; i < e; ++i) f(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}
}  // namespace

extern "C" {

void* orc_load_scene(const char* path, char* err, int errlen) {
    try {
        auto obj = loadSceneXML(path);
        auto sc = std::dynamic_pointer_cast<Scene>(obj);
        if (!sc) throw std::runtime_error("root element is not a scene");
        return new OracleScene{sc};
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return nullptr;
    }
}

// One mesh primitive with an identity transform built from a triangle soup
// (n x 9 floats): the traversal micro-benchmark's scene.
void* orc_mesh_scene(const float* tris, int64_t ntri, char* err, int errlen) {
    try {
        PropertyList p;
        auto mesh = std::make_shared<Mesh>(p);
        mesh->positions.resize(ntri * 3);
        for (int64_t i = 0; i < ntri * 3; ++i) mesh->positions[i] = Vec3(tris[i * 3], tris[i * 3 + 1], tris[i * 3 + 2]);
        mesh->indices.resize(ntri * 3);
        for (int64_t i = 0; i < ntri * 3; ++i) mesh->indices[i] = (uint32_t)i;
        mesh->activate();
        auto prim = std::make_shared<Primitive>(p);
        prim->addChild(mesh);
        prim->activate();
        auto sc = std::make_shared<Scene>(p);
        sc->addChild(prim);
        sc->buildTLAS();
        return new OracleScene{sc};
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return nullptr;
    }
}

void orc_free_scene(void* s) { delete (OracleScene*)s; }

// out: width, height, spp, maxDepth, integrator kind (0 path, 1 volpath), primitives, emitters
int orc_scene_info(void* s, int32_t* out) {
    auto& sc = *((OracleScene*)s)->scene;
    out[0] = sc.camera ? sc.camera->width : 0;
    out[1] = sc.camera ? sc.camera->height : 0;
    out[2] = sc.sampler ? sc.sampler->spp : 0;
    out[3] = sc.integrator ? sc.integrator->maxDepth : 0;
    out[4] = sc.integrator ? sc.integrator->kind : -1;
    out[5] = (int32_t)sc.prims.size();
    out[6] = (int32_t)sc.emitters.size();
    return 0;
}

// Renders passes [s0, s1) over the pixel window [x0,x1)x[y0,y1). film receives W*H*7
// floats per pixel (sum wL rgb, sum w, sum wL^2 rgb), accumulated on top of its content.
// stats: paths, rays (every scene.rayIntersect call).
int orc_render(void* s, int s0, int s1, int x0, int y0, int x1, int y1, int nthreads, float* film, uint64_t* stats,
               char* err, int errlen) {
    try {
        auto& sc = *((OracleScene*)s)->scene;
        Film f(sc.camera->width, sc.camera->height, sc.camera->filterObj);
        size_t n = (size_t)sc.camera->width * sc.camera->height * 7;
        for (size_t i = 0; i < n; ++i) f.sum[i].store(film[i], std::memory_order_relaxed);
        RenderStats st = renderPasses(sc, f, s0, s1, x0, y0, x1, y1, nthreads);
        for (size_t i = 0; i < n; ++i) film[i] = f.sum[i].load(std::memory_order_relaxed);
        if (stats) { stats[0] = st.paths; stats[1] = st.rays; }
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return -1;
    }
}

// As orc_render with the film in fixed point (Film::enableFixed): fsum receives W*H*4
// uint64 per pixel (sum wL rgb, sum w; units of 2^-24) and fsq W*H*3 floats (sum wL^2),
// both accumulated on top of their content (the integer sums modulo 2^64).
int orc_render_fixed(void* s, int s0, int s1, int x0, int y0, int x1, int y1, int nthreads, uint64_t* fsum, float* fsq,
                     uint64_t* stats, char* err, int errlen) {
    try {
        auto& sc = *((OracleScene*)s)->scene;
        Film f(sc.camera->width, sc.camera->height, sc.camera->filterObj);
        f.enableFixed();
        const size_t npix = (size_t)sc.camera->width * sc.camera->height;
        RenderStats st = renderPasses(sc, f, s0, s1, x0, y0, x1, y1, nthreads);
        for (size_t q = 0; q < npix; ++q) {
            for (int k = 0; k < 4; ++k) fsum[q * 4 + k] += f.fixedSum[q * 4 + k].load(std::memory_order_relaxed);
            for (int k = 0; k < 3; ++k) fsq[q * 3 + k] += f.sum[q * 7 + 4 + k].load(std::memory_order_relaxed);
        }
        if (stats) { stats[0] = st.paths; stats[1] = st.rays; }
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return -1;
    }
}

// Closest-hit (anyhit=0) or occlusion (anyhit=1) queries against the scene's TLAS.
// rays: n x 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax).
// Outputs (closest): t, u, v (barycentrics from the shape), prim (triangle index or -1),
// inst (original primitive index or -1); (any-hit) hit flag in inst (1/0).
// nodes/tris (optional): per-ray BVH4 node visits and triangle tests.
int orc_trace(void* s, const float* rays, int64_t n, int anyhit, int nthreads, float* t, float* u, float* v,
              int32_t* prim, int32_t* inst, uint32_t* nodes, uint32_t* tris) {
    auto& sc = *((OracleScene*)s)->scene;
    parallelFor(n, nthreads, [&](int64_t i) {
        const float* r = rays + i * 8;
        Ray ray(Vec3(r[0], r[1], r[2]), Vec3(r[4], r[5], r[6]), r[7]);
        ray.tMin = r[3];
        TraversalStats st;
        if (anyhit) {
            bool h = sc.occluded(ray, &st);
            inst[i] = h ? 1 : 0;
        } else {
            // closest hit without fillInteraction (bvh.cpp:38-60)
            float best = std::numeric_limits<float>::max();
            int bestInst = -1;
            SurfaceInteraction bestSi;
            auto leafFn = [&](int offset, int count) -> bool {
                bool hitLocal = false;
                for (int p = 0; p < count; ++p) {
                    SurfaceInteraction its;
                    if (sc.prims[offset + p]->rayIntersect(ray, its, false, &st)) {
                        if (its.t < best) {
                            ray.tMax = its.t;
                            best = its.t;
                            bestSi = its;
                            bestInst = sc.prims[offset + p]->originalIndex;
                            hitLocal = true;
                        }
                    }
                }
                return hitLocal;
            };
            bool h = traverseBVH4(sc.nodes4, ray, false, leafFn, &st);
            if (h) {
                t[i] = bestSi.t; u[i] = bestSi.uv.x; v[i] = bestSi.uv.y;
                // triangle index for meshes; analytic shapes have none (-1)
                bool isMesh = dynamic_cast<const Mesh*>(bestSi.primitive->shape.get()) != nullptr;
                prim[i] = isMesh ? (int32_t)bestSi.primIndex : -1;
                inst[i] = bestInst;
            } else {
                t[i] = Infinity; u[i] = 0; v[i] = 0; prim[i] = -1; inst[i] = -1;
            }
        }
        if (nodes) nodes[i] = (uint32_t)st.nodes;
        if (tris) tris[i] = (uint32_t)st.tris;
    });
    return 0;
}

// Full surface interaction for closest hits (p, n, dpdu, uv): out n x 11 floats.
int orc_trace_interaction(void* s, const float* rays, int64_t n, int nthreads, float* out, int32_t* inst) {
    auto& sc = *((OracleScene*)s)->scene;
    parallelFor(n, nthreads, [&](int64_t i) {
        const float* r = rays + i * 8;
        Ray ray(Vec3(r[0], r[1], r[2]), Vec3(r[4], r[5], r[6]), r[7]);
        ray.tMin = r[3];
        SurfaceInteraction si;
        float* o = out + i * 11;
        if (sc.rayIntersect(ray, si)) {
            o[0] = si.p.x; o[1] = si.p.y; o[2] = si.p.z;
            o[3] = si.n.x; o[4] = si.n.y; o[5] = si.n.z;
            o[6] = si.dpdu.x; o[7] = si.dpdu.y; o[8] = si.dpdu.z;
            o[9] = si.uv.x; o[10] = si.uv.y;
            inst[i] = si.primitive->originalIndex;
        } else {
            for (int k = 0; k < 11; ++k) o[k] = 0.f;
            inst[i] = -1;
        }
    });
    return 0;
}

// Camera rays for the render loop's first draws (integrator.h:92-125): n x 8 floats.
int orc_camera_rays(void* s, int spass, int64_t n, const int32_t* px, const int32_t* py, float* rays) {
    auto& sc = *((OracleScene*)s)->scene;
    const Camera& cam = *sc.camera;
    const int W = cam.width, H = cam.height;
    for (int64_t i = 0; i < n; ++i) {
        Sampler smp;
        smp.seed((uint64_t)py[i] * W + px[i] + (uint64_t)spass * ((uint64_t)W * H));
        Vec2 ps = smp.next2D();
        Vec2 pFilm(px[i] + ps.x, py[i] + ps.y);
        Vec2 camFilm(pFilm.x / W, 1.0f - pFilm.y / H);
        CameraSample cs;
        cs.pFilm = camFilm;
        cs.pLens = smp.next2D();
        const float channelRnd = smp.next1D();
        if (cam.hasChromaticAberration()) cs.lambdaOffset = channelRnd < 0.333333f ? 1.0f : (channelRnd < 0.666666f ? 0.0f : -1.0f);
        cs.time = smp.next1D();
        Ray r;
        cam.shootRay(cs, &r);
        float* o = rays + i * 8;
        o[0] = r.o.x; o[1] = r.o.y; o[2] = r.o.z; o[3] = r.tMin;
        o[4] = r.d.x; o[5] = r.d.y; o[6] = r.d.z; o[7] = r.tMax;
    }
    return 0;
}

// ------------------------------------------------------------------ known-answer helpers
float orc_fr_dielectric(float c, float a, float b) { return FrDielectric(c, a, b); }
void orc_fr_conductor(float c, const float* etaI, const float* etaT, const float* k, float* out) {
    FresnelConductor f(Color(etaI[0], etaI[1], etaI[2]), Color(etaT[0], etaT[1], etaT[2]), Color(k[0], k[1], k[2]));
    Color r = f.evaluate(c);
    out[0] = r.r; out[1] = r.g; out[2] = r.b;
}
int orc_refract(const float* wi, const float* n, float eta, float* wt) {
    Vec3 w;
    bool ok = Refract(Vec3(wi[0], wi[1], wi[2]), Vec3(n[0], n[1], n[2]), eta, &w);
    wt[0] = w.x; wt[1] = w.y; wt[2] = w.z;
    return ok ? 1 : 0;
}
float orc_roughness_to_alpha(float r) { return roughnessToAlpha(r); }
// op: 0 D(w), 1 G1(w), 2 G(wo, w2), 3 pdf(wo, w2), 4 sample_wh(wo, u) -> out[0..2]
float orc_ggx(int op, float alpha, const float* w, const float* w2, float* out) {
    TrowbridgeReitz d(alpha);
    Vec3 a(w[0], w[1], w[2]);
    Vec3 b = w2 ? Vec3(w2[0], w2[1], w2[2]) : Vec3();
    switch (op) {
        case 0: return d.D(a);
        case 1: return d.G1(a);
        case 2: return d.G(a, b);
        case 3: return d.pdf(a, b);
        case 4: { Vec3 h = d.sample_wh(a, Vec2(w2[0], w2[1])); out[0] = h.x; out[1] = h.y; out[2] = h.z; return 0.f; }
    }
    return 0.f;
}

// Lobe construction for the BxDF known-answer tests.
// kind: 0 Lambertian(R), 1 SpecularReflection(R, no-op Fresnel), 2 FresnelSpecular(R,T,ext,int),
// 3 MicrofacetReflection(R, alpha, no-op Fresnel), 4 MicrofacetFresnel(R,T,ext,int,alpha),
// 5 SmoothPlastic(Kd=R, Ks=T, eta=int), 6 RoughPlastic(Kd=R, Ks=T, eta=int, alpha),
// 7 SpecularTransmission(T, ext, int), 8 MicrofacetReflection(R, alpha, conductor(1, eta, k))
// p: R(3), T(3), etaExt, etaInt, alpha, condEta(3), condK(3)
static BxDF* makeLobe(int kind, const float* p, Arena& a) {
    Color R(p[0], p[1], p[2]), T(p[3], p[4], p[5]);
    float ext = p[6], in = p[7], alpha = p[8];
    switch (kind) {
        case 0: return a.create<Lambertian>(R);
        case 1: return a.create<SpecularReflection>(R, a.create<FresnelNoOp>());
        case 2: return a.create<FresnelSpecular>(R, T, ext, in);
        case 3: return a.create<MicrofacetReflection>(R, a.create<TrowbridgeReitz>(alpha), a.create<FresnelNoOp>());
        case 4: return a.create<MicrofacetFresnel>(R, T, ext, in, a.create<TrowbridgeReitz>(alpha));
        case 5: return a.create<SmoothPlastic>(R, T, in);
        case 6: return a.create<RoughPlastic>(R, T, in, a.create<TrowbridgeReitz>(alpha));
        case 7: return a.create<SpecularTransmission>(T, ext, in);
        case 8: return a.create<MicrofacetReflection>(R, a.create<TrowbridgeReitz>(alpha),
                                                      a.create<FresnelConductor>(Color(1.f), Color(p[9], p[10], p[11]), Color(p[12], p[13], p[14])));
    }
    return nullptr;
}
// Evaluates f (3 floats) and pdf of a lobe in its local frame.
int orc_bxdf_eval(int kind, const float* p, const float* wo, const float* wi, float* f, float* pdf) {
    Arena a;
    BxDF* b = makeLobe(kind, p, a);
    if (!b) return -1;
    Vec3 o(wo[0], wo[1], wo[2]), i(wi[0], wi[1], wi[2]);
    Color c = b->f(o, i);
    f[0] = c.r; f[1] = c.g; f[2] = c.b;
    *pdf = b->pdf(o, i);
    return 0;
}
// Samples a lobe; out: wi(3), f(3), pdf, type. pdf is preset to -1 to expose "not written".
int orc_bxdf_sample(int kind, const float* p, const float* wo, const float* u, float uc, float* wi, float* f, float* pdf, int* type) {
    Arena a;
    BxDF* b = makeLobe(kind, p, a);
    if (!b) return -1;
    Vec3 o(wo[0], wo[1], wo[2]), w;
    float pd = -1.f;
    BxDFType st = BxDFType(0);
    Color c = b->sample(o, w, Vec2(u[0], u[1]), uc, pd, &st);
    wi[0] = w.x; wi[1] = w.y; wi[2] = w.z;
    f[0] = c.r; f[1] = c.g; f[2] = c.b;
    *pdf = pd;
    *type = (int)st;
    return 0;
}
// Warps: op 0 disk (2 outputs), 1 uniform sphere, 2 uniform hemisphere, 3 cosine hemisphere,
// 4 cosine-hemisphere pdf of (u[0],u[1],u[2]) -> out[0], 5 polygon with (int)u[2] blades
// (2 outputs)
void orc_warp(int op, const float* u, float* out) {
    Vec2 s(u[0], u[1]);
    Vec3 r;
    switch (op) {
        case 0: { Vec2 d = warp::squareToUniformDisk(s); out[0] = d.x; out[1] = d.y; return; }
        case 1: r = warp::squareToUniformSphere(s); break;
        case 2: r = warp::squareToUniformHemisphere(s); break;
        case 3: r = warp::squareToCosineHemisphere(s); break;
        case 4: out[0] = warp::squareToCosineHemispherePdf(Vec3(u[0], u[1], u[2])); return;
        case 5: { Vec2 d = warp::squareToUniformPolygon(s, (int)u[2]); out[0] = d.x; out[1] = d.y; return; }
    }
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
// PCG32 stream: seeds with (initstate, initseq) and writes n uint32 draws.
void orc_pcg32(uint64_t initstate, uint64_t initseq, int n, uint32_t* out) {
    PCG32 r(initstate, initseq);
    for (int i = 0; i < n; ++i) out[i] = r.nextUInt();
}
uint64_t orc_splitmix64(uint64_t x) { return splitMix64(x); }
// Sampler seeded like the render loop (splitMix64 of the key); n floats.
void orc_sampler_floats(uint64_t key, int n, float* out) {
    Sampler s;
    s.seed(key);
    for (int i = 0; i < n; ++i) out[i] = s.next1D();
}
// Frame from a normal: out x(3), y(3), z(3)
void orc_frame(const float* n, float* out) {
    Frame f = Frame::fromNormal(Vec3(n[0], n[1], n[2]));
    float v[9] = {f.x.x, f.x.y, f.x.z, f.y.x, f.y.y, f.y.z, f.z.x, f.z.y, f.z.z};
    std::memcpy(out, v, sizeof(v));
}
// Shape known answers in object space. shape: 0 sphere(radius=p[0]), 1 cube(extents p[0..2]).
// out: hit, t, p(3), n(3)
int orc_shape_hit(int shape, const float* p, const float* ray, float* out) {
    PropertyList pl;
    std::unique_ptr<Shape> sh;
    if (shape == 0) { pl.f["radius"] = p[0]; sh = std::make_unique<Sphere>(pl); }
    else { pl.v3["extents"] = Vec3(p[0], p[1], p[2]); sh = std::make_unique<Cube>(pl); }
    Ray r(Vec3(ray[0], ray[1], ray[2]), Vec3(ray[4], ray[5], ray[6]), ray[7]);
    r.tMin = ray[3];
    SurfaceInteraction si;
    bool h = sh->rayIntersect(r, si, false, nullptr);
    out[0] = h ? 1.f : 0.f;
    if (h) {
        sh->fillInteraction(r, si);
        out[1] = si.t; out[2] = si.p.x; out[3] = si.p.y; out[4] = si.p.z; out[5] = si.n.x; out[6] = si.n.y; out[7] = si.n.z;
    }
    SurfaceInteraction dummy;
    out[8] = sh->pdfSurface(Vec3(10.f, 0.f, 0.f), dummy);
    return 0;
}
// Slab test of bounds.h:244-264: out t0, t1; returns hit
int orc_bounds_hit(const float* lo, const float* hi, const float* ray, float* out) {
    Bounds3 b(Vec3(lo[0], lo[1], lo[2]), Vec3(hi[0], hi[1], hi[2]));
    Ray r(Vec3(ray[0], ray[1], ray[2]), Vec3(ray[4], ray[5], ray[6]), ray[7]);
    return BoundsIntersect(b, r, &out[0], &out[1]) ? 1 : 0;
}
// Perspective camera ray for a film sample (perspective.cpp:15-32); out o(3), d(3)
void orc_perspective(float fov, int w, int h, float fx, float fy, float* out) {
    PropertyList pl;
    pl.f["fov"] = fov; pl.i["width"] = w; pl.i["height"] = h;
    Camera c(pl, 0);
    CameraSample cs;
    cs.pFilm = Vec2(fx, fy);
    Ray r;
    c.shootRay(cs, &r);
    out[0] = r.o.x; out[1] = r.o.y; out[2] = r.o.z; out[3] = r.d.x; out[4] = r.d.y; out[5] = r.d.z;
}
// Homogeneous medium sampling with explicit uniforms (homogeneous.cpp:32-63).
// in: sigma_a(3), sigma_s(3), tmax, u0, u1, d(3); out: weight(3), scattered, t
void orc_medium_sample(const float* in, float* out) {
    PropertyList pl;
    pl.c["sigma_a"] = Color(in[0], in[1], in[2]);
    pl.c["sigma_s"] = Color(in[3], in[4], in[5]);
    HomogeneousMedium m(pl);
    Ray r(Vec3(0.f), Vec3(in[9], in[10], in[11]), in[6]);
    Arena a;
    MediumInteraction mi;
    Color w = m.sampleU(r, in[7], in[8], a, mi);
    float t = mi.isValid() ? (mi.p - r.o).length() / r.d.length() : r.tMax;
    bool sm = mi.isValid();
    out[0] = w.r; out[1] = w.g; out[2] = w.b; out[3] = sm ? 1.f : 0.f; out[4] = t;
}
// HG phase: op 0 p(wo, wi) -> return; op 1 sample(wo, u) -> wi in out, returns value
float orc_hg(int op, float g, const float* wo, const float* x, float* out) {
    HGPhase h(g);
    Vec3 o(wo[0], wo[1], wo[2]);
    if (op == 0) return h.p(o, Vec3(x[0], x[1], x[2]));
    Vec3 wi;
    float v = h.sample(o, &wi, Vec2(x[0], x[1]));
    out[0] = wi.x; out[1] = wi.y; out[2] = wi.z;
    return v;
}

}  // extern "C"

// AnimatedTransform::interpolate (animated.cpp:29-47) between two affine matrices given
// row-major 4x4; out: the interpolated 3x4 matrix and its inverse (row-major).
extern "C" void orc_motion_interpolate(const float* a, const float* b, float time, float* out, float* outInv) {
    orc::Mat4 ma, mb;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) { ma.c[c][r] = a[4 * r + c]; mb.c[c][r] = b[4 * r + c]; }
    orc::AnimatedTransform at;
    at.set(orc::Transform(ma, orc::Mat4()), orc::Transform(mb, orc::Mat4()));
    orc::Transform t = at.interpolate(time);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) { out[4 * r + c] = t.m.c[c][r]; outInv[4 * r + c] = t.mInv.c[c][r]; }
}
