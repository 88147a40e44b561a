// gnd_host_*: C entry points of the host scene framework.
#include <cstring>
#include <string>

#include "hscene.h"

namespace gnd {
void setLastError(const std::string& msg);
}

namespace gndh {
struct HostScene {
    std::shared_ptr<Scene> scene;
};

template <typename F>
static gnd_status hguard(gnd_status failCode, F&& f) {
    try {
        f();
        return GND_OK;
    } catch (const std::bad_alloc&) {
        gnd::setLastError("host allocation failed");
        return GND_ERR_OOM;
    } catch (const std::exception& e) {
        gnd::setLastError(e.what());
        return failCode;
    }
}
}  // namespace gndh

using namespace gndh;

extern "C" {

gnd_status gnd_host_load_xml_ex(const char* path, int32_t flags, gnd_host_scene** out) {
    return hguard(GND_ERR_PARSE, [&]() {
        if (!path || !out) throw std::runtime_error("null argument");
        if (flags & ~GND_HOST_DEVICE_BLAS) throw std::runtime_error("unknown load flags");
        auto obj = loadFromXML(path, /*deferPreprocess=*/true, (flags & GND_HOST_DEVICE_BLAS) != 0);
        auto sc = std::dynamic_pointer_cast<Scene>(obj);
        if (!sc) throw std::runtime_error("root element is not a <scene>");
        *out = reinterpret_cast<gnd_host_scene*>(new HostScene{sc});
    });
}

gnd_status gnd_host_load_xml(const char* path, gnd_host_scene** out) { return gnd_host_load_xml_ex(path, 0, out); }

gnd_status gnd_host_from_triangles_ex(const float* tris, int64_t ntri, int32_t flags, gnd_host_scene** out) {
    return hguard(GND_ERR_INVALID, [&]() {
        if (!out || (ntri > 0 && !tris) || ntri < 0) throw std::runtime_error("bad triangle soup arguments");
        if (flags & ~GND_HOST_DEVICE_BLAS) throw std::runtime_error("unknown load flags");
        PropertyList p;
        auto sc = std::make_shared<Scene>(p);
        auto shape = std::dynamic_pointer_cast<ShapeObj>(std::shared_ptr<GndObject>(GndFactory::getInstance()->createInstance("mesh", p)));
        shape->positions.resize((size_t)ntri * 3);
        for (int64_t i = 0; i < ntri * 3; ++i) shape->positions[i] = gnd::v3(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
        auto prim = std::dynamic_pointer_cast<PrimitiveObj>(std::shared_ptr<GndObject>(GndFactory::getInstance()->createInstance("primitive", p)));
        prim->addChild(shape);
        prim->activate();
        sc->addChild(prim);
        sc->deviceBlas = (flags & GND_HOST_DEVICE_BLAS) != 0;
        sc->build();
        *out = reinterpret_cast<gnd_host_scene*>(new HostScene{sc});
    });
}

gnd_status gnd_host_from_triangles(const float* tris, int64_t ntri, gnd_host_scene** out) {
    return gnd_host_from_triangles_ex(tris, ntri, 0, out);
}

gnd_status gnd_host_scene_desc(const gnd_host_scene* s, const gnd_scene_desc** out) {
    return hguard(GND_ERR_INVALID, [&]() {
        if (!s || !out) throw std::runtime_error("null argument");
        *out = &reinterpret_cast<const HostScene*>(s)->scene->flat().desc;
    });
}

gnd_status gnd_host_free(gnd_host_scene* s) {
    delete reinterpret_cast<HostScene*>(s);
    return GND_OK;
}

}  // extern "C"
