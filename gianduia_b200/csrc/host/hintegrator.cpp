// The GPU integrator plugins: `path_gpu` and `volpath_gpu` (drop-ins for the reference's
// `path` and `volpath`, path.cpp:191 and volPath.cpp:301). They implement the
// reference's Integrator interface (integrator.h:18-40) on top of the C ABI:
//
//   preprocess(scene)  (called by Scene::activate, scene.cpp:61): creates the GPU context
//                      on first use and uploads the flattened scene (gnd_gpu_scene_upload)
//   render(scene)      (Scene::render, scene.cpp:73-75): renders the sampler's passes with
//                      gnd_gpu_render into the camera's film, reports every finished pass
//                      through the callback (integrator.h:148-149), and writes the film's
//                      EXR and PNG files (integrator.h:152-153)
//   cancel()           (integrator.h:22, from another thread or from the callback): the
//                      render stops after its current pass (gnd_gpu_cancel)
//
// Properties: maxDepth (path.cpp:9, volPath.cpp:12); device (CUDA ordinal, default 0);
// saveImages (default true: write the files as the reference does).
#include "hscene.h"

namespace gndh {

namespace {
void check(gnd_status s, const char* what) {
    if (s != GND_OK) throw std::runtime_error(std::string(what) + ": " + gnd_last_error());
}
}  // namespace

class GpuIntegratorBase : public Integrator {
public:
    GpuIntegratorBase(const PropertyList& p, int k) {
        kind = k;
        maxDepth = p.getInteger("maxDepth", 1000);   // path.cpp:9, volPath.cpp:12
        m_device = p.getInteger("device", 0);
        m_save = p.getBoolean("saveImages", true);
    }
    ~GpuIntegratorBase() override {
        if (m_ctx) {
            if (m_uploaded) gnd_gpu_scene_free(m_ctx, m_scene);
            gnd_gpu_destroy(m_ctx);
        }
    }

    void preprocess(Scene* scene) override {
        if (!m_ctx) check(gnd_gpu_create(m_device, &m_ctx), "GPU integrator: gnd_gpu_create");
        if (m_uploaded) {
            check(gnd_gpu_scene_free(m_ctx, m_scene), "GPU integrator: gnd_gpu_scene_free");
            m_uploaded = false;
        }
        check(gnd_gpu_scene_upload(m_ctx, &scene->flat().desc, &m_scene), "GPU integrator: gnd_gpu_scene_upload");
        m_uploaded = true;
    }

    // integrator.h:49-155 (SamplerIntegrator::render), every pass on the GPU
    void render(Scene* scene) override {
        m_stopRequested = false;
        if (!m_uploaded) preprocess(scene);
        Film* film = scene->ensureFilm();
        film->clear();
        const int W = film->width(), H = film->height();
        std::vector<float> sums((size_t)W * H * 7, 0.0f);
        gnd_render_params p{};
        p.spp = scene->getSampler()->spp;
        p.first_pass = 0;
        p.max_depth = maxDepth;
        p.integrator = kind;
        p.width = W;
        p.height = H;
        // With a callback the passes run one after another and each is reported as the
        // reference's loop reports it; without one every pass shares the path pool (the
        // film sums are the same either way).
        p.batched = m_callback ? 0 : 1;
        p.callback = m_callback ? &GpuIntegratorBase::onPass : nullptr;
        p.user = this;
        m_film = film;
        const gnd_status rc = gnd_gpu_render(m_ctx, m_scene, &p, sums.data(), &m_stats);
        m_film = nullptr;
        if (rc != GND_OK && rc != GND_ERR_CANCELLED) check(rc, "GPU integrator: gnd_gpu_render");
        film->setSums(sums.data());
        film->resolve();
        if (m_save) {   // integrator.h:152-153
            film->saveEXR();
            film->savePNG();
        }
    }

    void cancel() override {
        m_stopRequested = true;
        if (m_ctx) gnd_gpu_cancel(m_ctx);
    }

private:
    // gnd_progress_fn: one finished pass; the film so far is resolved and reported
    // (integrator.h:148-149: film->resolve(); notifyUpdate(s, *film)).
    static void onPass(void* user, int32_t sampleIndex, const float* sums, int32_t, int32_t) {
        auto* self = static_cast<GpuIntegratorBase*>(user);
        self->m_film->setSums(sums);
        self->m_film->resolve();
        self->notifyUpdate(sampleIndex, *self->m_film);
    }

    int m_device = 0;
    bool m_save = true;
    gnd_gpu_ctx* m_ctx = nullptr;
    gnd_scene_id m_scene = 0;
    bool m_uploaded = false;
    Film* m_film = nullptr;
    gnd_render_stats m_stats{};
};

struct PathGpuIntegrator : GpuIntegratorBase {
    explicit PathGpuIntegrator(const PropertyList& p) : GpuIntegratorBase(p, 0) {}
};
struct VolPathGpuIntegrator : GpuIntegratorBase {
    explicit VolPathGpuIntegrator(const PropertyList& p) : GpuIntegratorBase(p, 1) {}
};

GND_REGISTER_CLASS(PathGpuIntegrator, "path_gpu")
GND_REGISTER_CLASS(VolPathGpuIntegrator, "volpath_gpu")
// Scene files written for the CPU integrators render unchanged on the GPU.
struct PathAlias : PathGpuIntegrator {
    explicit PathAlias(const PropertyList& p) : PathGpuIntegrator(p) {}
};
struct VolPathAlias : VolPathGpuIntegrator {
    explicit VolPathAlias(const PropertyList& p) : VolPathGpuIntegrator(p) {}
};
GND_REGISTER_CLASS(PathAlias, "path")
GND_REGISTER_CLASS(VolPathAlias, "volpath")

}  // namespace gndh
