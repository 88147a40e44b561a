// C++ driver of the GPU integrator plugins, as the reference's application drives its
// integrators (application.cpp:503-515, 641: Parser::loadFromXML -> Scene::activate ->
// Integrator::preprocess, then Scene::render -> Integrator::render), against the
// library's mirror of the reference's plugin headers (hscene.h). Built with g++ by
// tests/test_gpu_plugin.py and run on a GPU.
//
//   plugin_driver <scene.xml> [cancel_after]
//
// Loads the scene through the plugin factory (the scene file names `path`, `path_gpu`,
// `volpath` or `volpath_gpu`), renders it through Integrator::render with a progress
// callback, and compares the camera film with a direct gnd_gpu_render of the same passes:
// sum wL and sum w must be bit-equal, the resolved radiance must be their quotient, the
// callback must see every pass in order, and the EXR and PNG files must exist. With
// cancel_after = k the callback cancels the render after pass k, so the film must hold
// passes 0..k only. Prints one line of results; exit status 0 when every check holds.
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <string>
#include <vector>

#include "gnd_gpu.h"
#include "hscene.h"

static int fail(const std::string& m) {
    std::printf("FAIL %s\n", m.c_str());
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 2) return fail("usage: plugin_driver <scene.xml> [cancel_after]");
    const std::string path = argv[1];
    const int cancelAfter = argc > 2 ? std::atoi(argv[2]) : -1;
    std::shared_ptr<gndh::Scene> scene;
    try {
        // parser.cpp:220-235 + scene.cpp:46-62: preprocess uploads the scene
        scene = std::dynamic_pointer_cast<gndh::Scene>(gndh::loadFromXML(path, /*deferPreprocess=*/false));
    } catch (const std::exception& e) {
        return fail(std::string("load: ") + e.what());
    }
    if (!scene) return fail("the root element is not a scene");
    auto integ = scene->getIntegrator();
    const int spp = scene->getSampler()->spp;
    std::vector<int> seen;
    bool sizeOk = true;
    integ->setCallback([&](int sampleIndex, const gndh::Film& film) {
        seen.push_back(sampleIndex);
        sizeOk = sizeOk && film.width() == scene->getCamera()->width && film.height() == scene->getCamera()->height;
        if (sampleIndex == cancelAfter) integ->cancel();
    });
    try {
        scene->render();   // scene.cpp:73-75
    } catch (const std::exception& e) {
        return fail(std::string("render: ") + e.what());
    }
    const int passes = cancelAfter >= 0 ? cancelAfter + 1 : spp;
    const gndh::Film* film = scene->getCamera()->getFilm();
    if (!film) return fail("no film");
    if ((int)seen.size() != passes) return fail("callback saw " + std::to_string(seen.size()) + " passes");
    for (int k = 0; k < passes; ++k)
        if (seen[k] != k) return fail("callback out of order");
    if (!sizeOk) return fail("callback film size");

    // the same passes through the C ABI
    gnd_host_scene* hs = nullptr;
    gnd_gpu_ctx* ctx = nullptr;
    gnd_scene_id sid = 0;
    const gnd_scene_desc* desc = nullptr;
    if (gnd_host_load_xml(path.c_str(), &hs) || gnd_host_scene_desc(hs, &desc) || gnd_gpu_create(0, &ctx) ||
        gnd_gpu_scene_upload(ctx, desc, &sid))
        return fail(std::string("C ABI setup: ") + gnd_last_error());
    const int W = film->width(), H = film->height();
    std::vector<float> direct((size_t)W * H * 7, 0.0f);
    gnd_render_params p{};
    p.spp = passes;
    p.integrator = -1;
    p.batched = 1;
    gnd_render_stats st{};
    if (gnd_gpu_render(ctx, sid, &p, direct.data(), &st)) return fail(std::string("gnd_gpu_render: ") + gnd_last_error());
    size_t diff = 0, resolveDiff = 0;
    double wsum = 0.0;
    const std::vector<float>& sums = film->sums();
    for (size_t q = 0; q < (size_t)W * H; ++q) {
        for (int k = 0; k < 4; ++k)
            if (sums[q * 7 + k] != direct[q * 7 + k]) ++diff;
        const float w = direct[q * 7 + 3];
        wsum += w;
        const float inv = 1.0f / w;
        const gndh::V3 e = w > 0.0f ? gnd::v3(direct[q * 7] * inv, direct[q * 7 + 1] * inv, direct[q * 7 + 2] * inv)
                                    : gnd::v3s(0.0f);
        const gndh::V3& r = film->getPixel((int)(q % W), (int)(q / W));
        if (r.x != e.x || r.y != e.y || r.z != e.z) ++resolveDiff;
    }
    const std::filesystem::path dir = std::filesystem::path(path).parent_path();
    const std::string stem = std::filesystem::path(path).stem().string();
    const bool files = std::filesystem::exists(dir / (stem + ".exr")) && std::filesystem::exists(dir / (stem + ".png"));
    std::printf("passes=%d spp=%d paths=%lld sum_w=%.1f sum_diff=%zu resolve_diff=%zu files=%d\n", passes, spp,
                (long long)st.paths, wsum, diff, resolveDiff, files ? 1 : 0);
    gnd_gpu_scene_free(ctx, sid);
    gnd_gpu_destroy(ctx);
    gnd_host_free(hs);
    if (st.paths != (int64_t)W * H * passes) return fail("direct render paths");
    if (diff) return fail("film sums differ from gnd_gpu_render");
    if (resolveDiff) return fail("resolved radiance");
    if (!files) return fail("EXR / PNG not written");
    if (wsum <= 0.0) return fail("empty film");
    std::printf("OK\n");
    return 0;
}
