// Oracle (test infrastructure only): integrators and render loop of the reference.
#pragma once
#include "oscene.h"

namespace orc {

struct RenderStats { uint64_t paths = 0, rays = 0; };

Color LiPath(const Scene& scene, const Ray& primary, Sampler& sampler, Arena& arena, int maxDepth, RenderStats& st);
Color LiVolPath(const Scene& scene, const Ray& primary, Sampler& sampler, Arena& arena, int maxDepth, RenderStats& st);
RenderStats renderPasses(const Scene& scene, Film& film, int s0, int s1, int x0, int y0, int x1, int y1, int nthreads);

}  // namespace orc
