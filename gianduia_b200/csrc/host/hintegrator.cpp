// The GPU integrator plugins: `path_gpu` and `volpath_gpu` (drop-ins for the reference's
// `path` and `volpath`, path.cpp:191 and volPath.cpp:301). They implement the
// reference's Integrator interface (integrator.h:18-40) on top of the C ABI.
#include "hscene.h"

namespace gndh {

class GpuIntegratorBase : public Integrator {
public:
    GpuIntegratorBase(const PropertyList& p, int k) {
        kind = k;
        maxDepth = p.getInteger("maxDepth", 1000);   // path.cpp:9, volPath.cpp:12
    }
    void preprocess(Scene*) override {}
    void render(Scene*) override {
        throw std::runtime_error("render through the scene plugin requires a GPU context; use gnd_gpu_render");
    }
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
