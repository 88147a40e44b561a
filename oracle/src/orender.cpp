// Oracle (test infrastructure only): the reference's `path` and `volpath` Li loops and
// its progressive render loop (one pass per sample, rows spread over threads),
// restated on the CPU. This is the image checker and the timed CPU baseline.
#include "orender.h"
#include <thread>

namespace orc {

static inline float powerHeuristic(int nf, float fPdf, int ng, float gPdf) {
    float f = nf * fPdf, g = ng * gPdf;
    float denom = (f * f) + (g * g);
    return denom > 0.0f ? (f * f) / denom : 0.0f;
}

// Environment light seen by an escaping ray (path.cpp:42-55, volPath.cpp:124-141): MIS
// against the environment's pdf, which the reference evaluates from the origin
// (a default SurfaceInteraction) towards r.o + 1e5 r.d.
static bool envMiss(const Scene& scene, const Ray& r, bool specularBounce, float pdfPrev, float nL, Color& Le, float& w) {
    if (!scene.envMap) return false;
    Le = scene.envMap->eval(SurfaceInteraction(), r.d);
    if (Le.isBlack()) return false;
    w = 1.0f;
    if (!specularBounce) {
        SurfaceInteraction envIsect;
        envIsect.p = r.o + r.d * 1e5f;
        envIsect.n = -r.d;
        float envPdf = scene.envMap->pdf(SurfaceInteraction(), envIsect);
        float pEnv = envPdf * (1.0f / nL);
        w = powerHeuristic(1, pdfPrev, 1, pEnv);
    }
    return true;
}

// path.cpp:12-181 (AOVs are not part of this restatement)
Color LiPath(const Scene& scene, const Ray& primary, Sampler& sampler, Arena& arena, int maxDepth, RenderStats& st) {
    Color L(0.0f), tp(1.0f);
    Ray r = primary;
    int bounces = 0, nullBounces = 0;
    bool specularBounce = true;
    float pdfPrev = 1.0f;
    Vec3 lastScatter = primary.o;
    const float nL = (float)scene.emitters.size();
    while (bounces < maxDepth) {
        SurfaceInteraction isect;
        st.rays++;
        bool hit = scene.rayIntersect(r, isect);
        if (!hit) {
            Color Le;
            float w;
            if (envMiss(scene, r, specularBounce, pdfPrev, nL, Le, w)) L += tp * Le * w;
            break;
        }
        isect.primitive->material->computeScatteringFunctions(isect, arena);
        if (isect.primitive->emitter) {
            const Emitter* em = isect.primitive->emitter.get();
            bool skip = (bounces == 0 && !isect.bsdf);
            if (!skip) {
                Color Le = em->eval(isect, -r.d);
                if (!Le.isBlack()) {
                    float w = 1.0f;
                    if (!specularBounce) {
                        SurfaceInteraction ref; ref.p = lastScatter;
                        float lightPdf = em->pdf(ref, isect);
                        float pl = lightPdf * (1.0f / nL);
                        w = powerHeuristic(1, pdfPrev, 1, pl);
                    }
                    L += tp * Le * w;
                }
            }
        }
        if (!isect.bsdf) {
            if (nullBounces++ > 100) break;
            Ray nr(isect.p, r.d);
            nr.time = isect.time;
            r = nr;
            continue;
        }
        // next event estimation, path.cpp:104-151
        float lightSelectPdf = 1.0f / nL;
        const Emitter* em = scene.randomEmitter(sampler.next1D());
        SurfaceInteraction lightIsect;
        float lightPdf = 0.0f;
        Ray shadowRay;
        Color Li = em->sample(isect, sampler.next2D(), lightIsect, lightPdf, shadowRay);
        Li /= lightSelectPdf;
        if (lightPdf > 1e-6f && !Li.isBlack()) {
            bool occ = false;
            Ray tr = shadowRay;
            for (;;) {
                SurfaceInteraction sh;
                st.rays++;
                if (!scene.rayIntersect(tr, sh)) break;
                sh.primitive->material->computeScatteringFunctions(sh, arena);
                if (sh.bsdf != nullptr) { occ = true; break; }
                // tr.tMax already holds the hit distance here (path.cpp:124-131)
                float nextTmax = tr.tMax - (sh.p - tr.o).length();
                Ray nr(sh.p, tr.d);
                nr.tMax = nextTmax;
                nr.time = sh.time;
                tr = nr;
            }
            if (!occ) {
                Vec3 wi = Normalize(lightIsect.p - isect.p);
                float bsdfPdf = isect.bsdf->pdf(-r.d, wi);
                Color f = isect.bsdf->f(-r.d, wi);
                if (!f.isBlack() && bsdfPdf > 1e-6f) {
                    float pl = lightPdf * lightSelectPdf;
                    float pb = em->isDelta() ? 0.0f : bsdfPdf;
                    float wl = powerHeuristic(1, pl, 1, pb);
                    L += tp * f * Li * std::abs(Dot(isect.n, wi)) * wl;
                }
            }
        }
        // BSDF sampling, path.cpp:153-172
        Vec3 wi;
        BxDFType sampledType = BxDFType(0);
        Vec2 u2 = sampler.next2D();
        float u1 = sampler.next1D();
        Color fcos = isect.bsdf->sample(-r.d, &wi, u2, u1, &pdfPrev, &sampledType);
        if (fcos.isBlack() || pdfPrev <= 1e-6f) break;
        specularBounce = (sampledType & BSDF_SPECULAR) != 0;
        tp *= fcos;
        if (bounces > 2) {
            float q = std::max(0.05f, std::min(tp.luminance(), 0.99f));
            if (sampler.next1D() > q) break;
            tp /= q;
        }
        lastScatter = isect.p;
        Ray nr(isect.p, wi);
        nr.time = isect.time;
        r = nr;
        bounces++;
    }
    return L;
}

// volPath.cpp:293-298
static const Medium* nextMedium(const Vec3& wo, const Vec3& wi, const Medium* cur, const SurfaceInteraction& si) {
    if (Dot(wi, si.n) > 0.0f) return Dot(wo, si.n) > 0.0f ? cur : si.mediumInterface.outside;
    return Dot(wo, si.n) > 0.0f ? si.mediumInterface.inside : cur;
}

// volPath.cpp:261-291
static Color evaluateTr(const Scene& scene, Ray sr, const Vec3& lightP, Arena& arena, RenderStats& st) {
    Color Tr(1.0f);
    Ray r = sr;
    for (;;) {
        SurfaceInteraction isect;
        st.rays++;
        bool hit = scene.rayIntersect(r, isect);
        if (r.medium) {
            Ray trRay = r;
            trRay.tMax = hit ? isect.t : r.tMax;
            Tr *= r.medium->Tr(trRay);
        }
        if (Tr.isBlack()) return Tr;
        if (!hit) break;
        isect.primitive->material->computeScatteringFunctions(isect, arena);
        if (isect.bsdf != nullptr) return Color(0.0f);
        const Medium* m = isect.getMedium(r.d);
        Ray nr(isect.p, r.d);
        nr.medium = m;
        nr.tMin = Epsilon;
        nr.tMax = (isect.p - lightP).length() - Epsilon;
        nr.time = isect.time;
        r = nr;
    }
    return Tr;
}

// volPath.cpp:15-252
Color LiVolPath(const Scene& scene, const Ray& primary, Sampler& sampler, Arena& arena, int maxDepth, RenderStats& st) {
    Color L(0.0f), tp(1.0f);
    Ray r = primary;
    int bounces = 0, surfaceBounces = 0, volumeBounces = 0, nullBounces = 0;
    float pdfPrev = 1.0f;
    bool specularBounce = true;
    Vec3 lastScatter = primary.o;
    const float nL = (float)scene.emitters.size();
    while (bounces < maxDepth) {
        SurfaceInteraction isect;
        st.rays++;
        bool hitSurface = scene.rayIntersect(r, isect);
        MediumInteraction mi;
        if (r.medium) tp *= r.medium->sample(r, sampler, arena, mi);
        if (mi.isValid()) {
            tp *= mi.sigma_s;
            if (tp.isBlack()) break;
            float lightSelectPdf = 1.0f / nL;
            const Emitter* em = scene.randomEmitter(sampler.next1D());
            SurfaceInteraction ref;
            ref.p = mi.p;
            SurfaceInteraction lightIsect;
            float lightPdf = 0.0f;
            Ray shadowRay;
            Color Li = em->sample(ref, sampler.next2D(), lightIsect, lightPdf, shadowRay);
            Li /= lightSelectPdf;
            if (lightPdf > 1e-6f && !Li.isBlack()) {
                shadowRay.medium = mi.medium;
                Color Tr = evaluateTr(scene, shadowRay, lightIsect.p, arena, st);
                if (!Tr.isBlack()) {
                    Vec3 wi = Normalize(lightIsect.p - mi.p);
                    float phasePdf = mi.phase->p(mi.wo, wi);
                    if (phasePdf > 1e-6f) {
                        float pl = lightPdf * lightSelectPdf;
                        float pp = em->isDelta() ? 0.0f : phasePdf;
                        float wl = powerHeuristic(1, pl, 1, pp);
                        L += tp * phasePdf * Li * wl * Tr;
                    }
                }
            }
            Vec3 wi;
            pdfPrev = mi.phase->sample(mi.wo, &wi, sampler.next2D());
            specularBounce = false;
            const Medium* prevMedium = r.medium;
            float prevTime = r.time;
            lastScatter = mi.p;
            Ray nr(mi.p, wi);
            nr.medium = prevMedium;
            nr.time = prevTime;
            r = nr;
            if (volumeBounces > 6) {
                float q = std::max(0.05f, std::min(tp.luminance(), 0.99f));
                if (sampler.next1D() > q) break;
                tp /= q;
            }
            bounces++;
            volumeBounces++;
            continue;
        }
        const Medium* curMedium = r.medium;
        if (!hitSurface) {
            Color Le;
            float w;
            if (envMiss(scene, r, specularBounce, pdfPrev, nL, Le, w)) L += tp * Le * w;
            break;
        }
        isect.primitive->material->computeScatteringFunctions(isect, arena);
        if (isect.primitive->emitter) {
            const Emitter* em = isect.primitive->emitter.get();
            bool skip = (bounces == 0 && !isect.bsdf);
            if (!skip) {
                Color Le = em->eval(isect, -r.d);
                if (!Le.isBlack()) {
                    float w = 1.0f;
                    if (!specularBounce) {
                        SurfaceInteraction ref; ref.p = lastScatter;
                        float lightPdf = em->pdf(ref, isect);
                        float pl = lightPdf * (1.0f / nL);
                        w = powerHeuristic(1, pdfPrev, 1, pl);
                    }
                    L += tp * Le * w;
                }
            }
        }
        if (!isect.bsdf) {
            if (nullBounces++ > 100) break;
            const Medium* m = isect.getMedium(r.d);
            Ray nr(isect.p, r.d);
            nr.medium = m;
            nr.time = isect.time;
            r = nr;
            continue;
        }
        float lightSelectPdf = 1.0f / nL;
        const Emitter* em = scene.randomEmitter(sampler.next1D());
        SurfaceInteraction lightIsect;
        float lightPdf = 0.0f;
        Ray shadowRay;
        Color Li = em->sample(isect, sampler.next2D(), lightIsect, lightPdf, shadowRay);
        Li /= lightSelectPdf;
        if (lightPdf > 1e-6f && !Li.isBlack()) {
            shadowRay.medium = nextMedium(-r.d, shadowRay.d, curMedium, isect);
            Color Tr = evaluateTr(scene, shadowRay, lightIsect.p, arena, st);
            if (!Tr.isBlack()) {
                Vec3 wi = Normalize(lightIsect.p - isect.p);
                float bsdfPdf = isect.bsdf->pdf(-r.d, wi);
                Color f = isect.bsdf->f(-r.d, wi);
                if (!f.isBlack() && bsdfPdf > 1e-6f) {
                    float pl = lightPdf * lightSelectPdf;
                    float pb = em->isDelta() ? 0.0f : bsdfPdf;
                    float wl = powerHeuristic(1, pl, 1, pb);
                    L += tp * f * Li * std::abs(Dot(isect.n, wi)) * wl * Tr;
                }
            }
        }
        BxDFType sampledType = BxDFType(0);
        Vec3 wi;
        Vec2 u2 = sampler.next2D();
        float u1 = sampler.next1D();
        Color fcos = isect.bsdf->sample(-r.d, &wi, u2, u1, &pdfPrev, &sampledType);
        if (fcos.isBlack() || pdfPrev <= 1e-6f) break;
        specularBounce = (sampledType & BSDF_SPECULAR) != 0;
        tp *= fcos;
        Vec3 incident = -r.d;
        lastScatter = isect.p;
        Ray nr(isect.p, wi);
        nr.medium = nextMedium(incident, wi, curMedium, isect);
        nr.time = isect.time;
        r = nr;
        if (surfaceBounces > 2) {
            float q = std::max(0.05f, std::min(tp.luminance(), 0.99f));
            if (sampler.next1D() > q) break;
            tp /= q;
        }
        bounces++;
        surfaceBounces++;
    }
    return L;
}

// integrator.h:49-155: one pass per sample index s in [s0, s1); each pixel sample is
// seeded with y*W + x + s*W*H. Rows of the window [x0,x1)x[y0,y1) are spread over
// `nthreads` workers; per pass the film receives exactly one sample per pixel.
RenderStats renderPasses(const Scene& scene, Film& film, int s0, int s1, int x0, int y0, int x1, int y1, int nthreads) {
    const Camera& cam = *scene.camera;
    const int W = cam.width, H = cam.height;
    const int kind = scene.integrator->kind;
    const int maxDepth = scene.integrator->maxDepth;
    RenderStats total;
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    for (int s = s0; s < s1; ++s) {
        std::atomic<int> nextRow{y0};
        std::vector<RenderStats> per(nthreads);
        auto work = [&](int tid) {
            Sampler smp;
            Arena arena(1 << 18);
            RenderStats& st = per[tid];
            for (;;) {
                int y = nextRow.fetch_add(1);
                if (y >= y1) break;
                for (int x = x0; x < x1; ++x) {
                    arena.reset();
                    uint64_t pixelIdx = (uint64_t)y * W + x;
                    uint64_t globalIdx = pixelIdx + (uint64_t)s * ((uint64_t)W * H);
                    smp.seed(globalIdx);
                    Vec2 ps = smp.next2D();
                    Vec2 pFilm(x + ps.x, y + ps.y);
                    Vec2 camFilm(pFilm.x / W, 1.0f - pFilm.y / H);
                    CameraSample cs;
                    cs.pFilm = camFilm;
                    cs.pLens = smp.next2D();
                    // integrator.h:103-121: one colour channel per sample under chromatic aberration
                    float channelRnd = smp.next1D();
                    int channel;
                    if (!cam.hasChromaticAberration()) {
                        channel = -1;
                        cs.lambdaOffset = 0.0f;
                    } else if (channelRnd < 0.333333f) {
                        channel = 0;
                        cs.lambdaOffset = 1.0f;
                    } else if (channelRnd < 0.666666f) {
                        channel = 1;
                        cs.lambdaOffset = 0.0f;
                    } else {
                        channel = 2;
                        cs.lambdaOffset = -1.0f;
                    }
                    cs.time = smp.next1D();
                    Ray ray;
                    float rayWeight = cam.shootRay(cs, &ray);
                    Color raw = kind == 0 ? LiPath(scene, ray, smp, arena, maxDepth, st)
                                          : LiVolPath(scene, ray, smp, arena, maxDepth, st);
                    raw = raw * rayWeight;
                    Color L(0.0f);
                    if (channel == -1) L = raw;
                    else if (channel == 0) L.r = raw.r * 3.0f;
                    else if (channel == 1) L.g = raw.g * 3.0f;
                    else L.b = raw.b * 3.0f;
                    if (L.hasNaNs()) L = Color(0.0f);
                    film.addSample(pFilm, L);
                    st.paths++;
                }
            }
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
        work(0);
        for (auto& t : th) t.join();
        for (auto& p : per) { total.paths += p.paths; total.rays += p.rays; }
    }
    return total;
}

}  // namespace orc
