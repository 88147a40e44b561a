// Host scene framework: the reference's plugin object model (GndObject, PropertyList,
// GND_REGISTER_CLASS, Scene, Primitive, shapes, materials, media, emitters, camera,
// filters, sampler, Integrator), producing the flattened device layout that the GPU
// integrators consume.
#pragma once
#include <atomic>
#include <cstdint>
#include <filesystem>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "gnd/layout.h"
#include "gnd/motion.h"
#include "gnd/vmath.h"
#include "gnd_gpu.h"

namespace gndh {

using gnd::V2;
using gnd::V3;

// ---------------------------------------------------------------- 4x4 matrices
// Column-major like glm::mat4: c[col][row].
struct Mat4 {
    float c[4][4];
    static Mat4 identity();
    Mat4 operator*(const Mat4& b) const;
    void mulVec(const float v[4], float out[4]) const;   // (c0*x + c1*y) + (c2*z + c3*w)
    Mat4 transpose() const;
    bool operator==(const Mat4& o) const;
    gnd::Xf34 toXf34() const;
};
Mat4 inverse(const Mat4& m);   // cofactor expansion

// transform.h:299-437: matrix and inverse composed step by step (parser: t = step * t)
struct Transform {
    Mat4 m = Mat4::identity(), mInv = Mat4::identity();
    Transform() = default;
    Transform(const Mat4& a, const Mat4& b) : m(a), mInv(b) {}
    Transform inverse() const { return Transform(mInv, m); }
    Transform operator*(const Transform& t) const { return Transform(m * t.m, t.mInv * mInv); }
    bool operator==(const Transform& o) const { return m == o.m; }
    V3 point(V3 p) const;
    V3 vector(V3 v) const;
    static Transform translate(V3 d);
    static Transform scale(float x, float y, float z);
    static Transform rotate(float degrees, V3 axis);
    static Transform lookAt(V3 pos, V3 target, V3 up);
};

struct Bounds {
    V3 lo{3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    V3 hi{-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    void grow(V3 p);
    void grow(const Bounds& b);
    V3 centroid() const { return lo * 0.5f + hi * 0.5f; }   // bounds.h:214-216
    float area() const;                                      // bounds.h:184-187
    int maxExtent() const;                                   // bounds.h:196-203
    Bounds transformed(const Transform& t) const;            // transform.h:356-363
};

// ---------------------------------------------------------------- properties
// propertyList.h:12-100
class PropertyList {
public:
    void setBoolean(const std::string& k, bool v) { b_[k] = v; }
    void setInteger(const std::string& k, int v) { i_[k] = v; }
    void setFloat(const std::string& k, float v) { f_[k] = v; }
    void setString(const std::string& k, const std::string& v) { s_[k] = v; }
    void setPoint3(const std::string& k, V3 v) { p3_[k] = v; }
    void setVector2(const std::string& k, V2 v) { v2_[k] = v; }
    void setPoint2(const std::string& k, V2 v) { p2_[k] = v; }
    void setVector3(const std::string& k, V3 v) { v3_[k] = v; }
    void setColor(const std::string& k, V3 v) { c_[k] = v; }
    void setTransform(const std::string& k, const Transform& v) { t_[k] = v; }
    bool hasColor(const std::string& k) const { return c_.count(k) > 0; }
    bool hasFloat(const std::string& k) const { return f_.count(k) > 0; }
    bool hasTransform(const std::string& k) const { return t_.count(k) > 0; }
    bool getBoolean(const std::string& k, bool d = false) const { return get(b_, k, d); }
    int getInteger(const std::string& k, int d = 0) const { return get(i_, k, d); }
    float getFloat(const std::string& k, float d = 0.f) const { return get(f_, k, d); }
    std::string getString(const std::string& k, const std::string& d = "") const { return get(s_, k, d); }
    V3 getVector3(const std::string& k, V3 d) const { return get(v3_, k, d); }
    V2 getVector2(const std::string& k, V2 d) const { return get(v2_, k, d); }
    V2 getPoint2(const std::string& k, V2 d) const { return get(p2_, k, d); }
    V3 getColor(const std::string& k, V3 d) const { return get(c_, k, d); }
    V3 getPoint3(const std::string& k, V3 d) const { return get(p3_, k, d); }
    Transform getTransform(const std::string& k, const Transform& d) const { return get(t_, k, d); }

private:
    template <typename M, typename V>
    static V get(const M& m, const std::string& k, const V& d) {
        auto it = m.find(k);
        return it == m.end() ? d : it->second;
    }
    std::map<std::string, bool> b_;
    std::map<std::string, int> i_;
    std::map<std::string, float> f_;
    std::map<std::string, std::string> s_;
    std::map<std::string, V3> p3_, v3_, c_;
    std::map<std::string, V2> v2_, p2_;
    std::map<std::string, Transform> t_;
};

// ---------------------------------------------------------------- object model
// object.h:11-23
enum EClassType { EScene, EPrimitive, EShape, ECamera, EIntegrator, ESampler, ETexture, EMaterial, EEmitter, EFilter, EMedium };
const char* classTypeToString(EClassType t);

class GndObject {
public:
    virtual ~GndObject() = default;
    virtual void addChild(std::shared_ptr<GndObject>) { throw std::runtime_error("GndObject::addChild() not implemented!"); }
    virtual void activate() {}
    virtual EClassType getClassType() const = 0;
    // directory of the scene file, for objects that read files (FileResolver::resolve)
    virtual void setBaseDir(const std::string&) {}
    void setName(const std::string& n) { m_name = n; }
    const std::string& getName() const { return m_name; }

protected:
    std::string m_name;
};

// fileResolver.h:11-41: the directory of the scene file being loaded and the name its
// outputs take (its stem), recorded by loadFromXML as Parser::loadFromXML records them
// (parser.cpp:220-223) before the scene is built.
// Process-wide like the reference's; a mutex makes loads on several threads safe, the
// values being those of the latest load to set them.
class FileResolver {
public:
    static void setBasePath(const std::filesystem::path& p);
    static void setOutputPath(const std::filesystem::path& p);
    static void setOutputName(const std::string& n);
    static std::filesystem::path getBasePath();
    static std::filesystem::path getOutputPath();
    static std::string getOutputName();
};

// factory.h:9-36
using ObjectFactory = std::function<std::unique_ptr<GndObject>(const PropertyList&)>;
class GndFactory {
public:
    static GndFactory* getInstance();
    void registerClass(const std::string& name, const ObjectFactory& f);
    std::unique_ptr<GndObject> createInstance(const std::string& name, const PropertyList& props);
    bool has(const std::string& name) const { return m_ctors.count(name) > 0; }

private:
    std::map<std::string, ObjectFactory> m_ctors;
};
#define GND_REGISTER_CLASS(Cls, XmlName)                                                                   \
    namespace {                                                                                          \
    struct Cls##_Factory {                                                                               \
        Cls##_Factory() {                                                                                \
            ::gndh::GndFactory::getInstance()->registerClass(                                            \
                XmlName, [](const ::gndh::PropertyList& p) -> std::unique_ptr<::gndh::GndObject> {       \
                    return std::make_unique<Cls>(p);                                                     \
                });                                                                                      \
        }                                                                                                \
    };                                                                                                   \
    Cls##_Factory global_##Cls##_Factory;                                                                \
    }

// Texture trees of a scene as the device reads them: nodes, image texels (rgba) and the
// node of each texture object already flattened.
struct TexTables {
    std::vector<gnd::TexNode> nodes;
    std::vector<float> texels;
    std::map<const void*, int32_t> done;
};

// Color texture description: constant_color / checkerboard_color live in the slot itself
// (rec); the other textures set rec.kind = kTexNode and flatten into a node tree.
struct ColorTexture : GndObject {
    gnd::ColorTex rec{};
    EClassType getClassType() const override { return ETexture; }
    // Appends this texture's node (after its inputs') to t and returns its index.
    int32_t flatten(TexTables& t) const;
    virtual gnd::TexNode node(TexTables& t) const;   // constant / checker leaf from rec
    virtual bool isNormalMap() const { return false; }
};
// Float texture: a constant, or (constant false) a texture tree whose nodes carry the
// value in every channel. `tree` is set for both, so a float texture can also be a node
// of another tree (the base of a float domain warp).
struct FloatTexture : GndObject {
    float value = 1.f;
    bool constant = true;
    std::shared_ptr<ColorTexture> tree;
    EClassType getClassType() const override { return ETexture; }
};

struct MediumObj : GndObject {
    gnd::Medium rec{};
    EClassType getClassType() const override { return EMedium; }
};

struct MaterialObj : GndObject {
    gnd::Material rec{};
    std::shared_ptr<ColorTexture> texA, texB;   // the texture objects of slots a and b
    std::shared_ptr<ColorTexture> roughTex, etaTex, kTex;   // non-constant roughness / eta / k
    std::shared_ptr<ColorTexture> normalTex, bumpTex;       // normal / bump map trees (material.h:36-44)
    std::shared_ptr<MediumObj> inside, outside;
    EClassType getClassType() const override { return EMaterial; }
    void addChild(std::shared_ptr<GndObject> c) override;
};

struct EmitterObj : GndObject {
    int32_t type = gnd::kEmitArea;
    gnd::ColorTex radiance{};      // area
    std::shared_ptr<ColorTexture> radianceTex;
    bool hasRadiance = false;
    // point / spot / directional (pointlight.cpp, spotlight.cpp, directional.cpp)
    V3 position{}, direction{}, color{};
    float cosTotal = 0.0f, cosFalloff = 0.0f;
    // environment map (environment.cpp): texels and sampling tables (gnd_scene_desc layout)
    std::string filename, baseDir;
    float strength = 1.0f;
    int envWidth = 0, envHeight = 0;
    std::vector<float> envTexels, envDist;
    float envMarginalIntegral = 0.0f;
    EClassType getClassType() const override { return EEmitter; }
    void addChild(std::shared_ptr<GndObject> c) override;
    void activate() override;
    void setBaseDir(const std::string& d) override { baseDir = d; }
    bool isInfiniteAreaLight() const { return type == gnd::kEmitEnv; }
};

// Motion record of a transform moving from `a` (time 0) to `b` (time 1): both decomposed
// (animated.cpp:18-21) and b's matrices; and the transform at time 0.5 (motion bounds).
gnd::InstMotion makeMotion(const Transform& a, const Transform& b);
Transform motionMid(const gnd::InstMotion& k);

// OpenEXR scanline image (NO, ZIPS or ZIP compression; HALF or FLOAT channels): the
// R, G, B channels as rgb floats, row-major (himage.cpp).
void readEXR(const std::string& path, int& width, int& height, std::vector<float>& rgb);
// TextureCache::load (textureCache.h:23-95): an image texture's texels as rgba floats, row 0
// the image's bottom row. OpenEXR through half precision (R, G, B; alpha 1); PNG (8 or
// 16 bit, grey, grey + alpha, RGB, RGBA; 16-bit samples keep their high byte) divided by
// 255, with the sRGB curve on every channel of 1-3 channel images and on RGB of RGBA ones.
// `channels` is the file's channel count.
void readTextureImage(const std::string& path, bool srgb, int& width, int& height, int& channels, std::vector<float>& rgba);

// Mesh geometry in the reference's de-indexed form (one vertex per face corner).
struct ShapeObj : GndObject {
    uint32_t kind = gnd::kShapeMesh;
    std::string filename;
    std::vector<V3> positions, normals;
    std::vector<V2> uvs;
    float radius = 1.f;
    V3 extents{1.f, 1.f, 1.f};
    int meshId = -1;      // assigned at flattening
    EClassType getClassType() const override { return EShape; }
    void activate() override;
    Bounds objectBounds() const;
    size_t numTris() const { return positions.size() / 3; }
};

struct PrimitiveObj : GndObject {
    Transform toWorld;
    Transform toWorldEnd;     // primitive.cpp:8: the transform at shutter time 1
    bool animated = false;    // toWorldEnd differs from toWorld (animated.cpp:16)
    std::shared_ptr<ShapeObj> shape;
    std::shared_ptr<MaterialObj> material;
    std::shared_ptr<EmitterObj> emitter;
    explicit PrimitiveObj(const PropertyList& p);
    EClassType getClassType() const override { return EPrimitive; }
    void addChild(std::shared_ptr<GndObject> c) override;
    void activate() override;
};

struct FilterObj : GndObject {
    int type = 0;   // 0 box, 1 gaussian
    float rx = 0.5f, ry = 0.5f, alpha = 2.f;
    EClassType getClassType() const override { return EFilter; }
};

// film.h:21-136: the image a render writes. The GPU integrators fill it from the device's
// per-pixel sums (sum wL rgb, sum w, sum wL^2 rgb: setSums) and resolve it as
// film.cpp:50-95 does; savePNG / saveEXR write <outputPath>/<outputName>.png / .exr as
// film.cpp:154-195 (the scene file's directory and stem, FileResolver).
class Film {
public:
    Film(int width, int height);
    void clear();
    // sums: width x height x 7 floats (the layout of gnd_gpu_render's film)
    void setSums(const float* sums);
    const std::vector<float>& sums() const { return m_sums; }
    // radiance = sum wL / sum w per pixel, 0 where no sample has weight
    void resolve();
    void setPixel(int x, int y, V3 c) { m_radiance[(size_t)y * m_width + x] = c; }
    const V3& getPixel(int x, int y) const { return m_radiance[(size_t)y * m_width + x]; }
    const std::vector<V3>& getRadiance() const { return m_radiance; }
    int width() const { return m_width; }
    int height() const { return m_height; }
    float aspectRatio() const { return (float)m_width / (float)m_height; }
    void savePNG() const { savePNG(outputName); }
    void saveEXR() const { saveEXR(outputName); }
    void savePNG(const std::string& relativeOutPath) const;   // sRGB, x255 + 0.5, clamped, truncated
    void saveEXR(const std::string& relativeOutPath) const;   // float RGB
    std::string outputPath = ".", outputName = "output";

private:
    int m_width, m_height;
    std::vector<float> m_sums;
    std::vector<V3> m_radiance;
};

struct CameraObj : GndObject {
    Transform toWorld;
    Transform toWorldEnd;     // camera.h:23
    bool animated = false;
    bool rollingShutter = false;                         // thinLens.cpp:28-30
    float scanDuration = 0.9f, exposureDuration = 0.1f;
    int width = 1280, height = 720;
    float fov = 45.f;
    // thin lens (thinLens.cpp:13-31); kind 0 is the pinhole `perspective` camera
    int kind = 0;
    float lensRadius = 0.0f, focalDistance = 10.0f, k1 = 0.0f, caAxial = 0.0f, caLateral = 0.0f;
    bool vignetting = false;
    int blades = 0;
    std::shared_ptr<FilterObj> filter;
    std::unique_ptr<Film> film;   // camera.h:72: created by Scene::activate
    explicit CameraObj(const PropertyList& p);
    EClassType getClassType() const override { return ECamera; }
    void addChild(std::shared_ptr<GndObject> c) override;
    // camera.h:32-39
    Film* getFilm() const { return film.get(); }
    int getWidth() const { return width; }
    int getHeight() const { return height; }
};

struct SamplerObj : GndObject {
    int spp = 1;
    explicit SamplerObj(const PropertyList& p) : spp(p.getInteger("spp", 1)) {}
    EClassType getClassType() const override { return ESampler; }
    size_t getSampleCount() const { return (size_t)spp; }   // sampler.h:21
};

class Scene;

// integrator.h:18-40: the plugin interface the GPU integrators implement.
class Integrator : public GndObject {
public:
    using RenderCallback = std::function<void(int sampleIndex, const Film& film)>;
    virtual ~Integrator() = default;
    virtual void render(Scene* scene) = 0;
    virtual void cancel() { m_stopRequested = true; }
    virtual void preprocess(Scene*) {}
    void setCallback(RenderCallback cb) { m_callback = std::move(cb); }
    EClassType getClassType() const override { return EIntegrator; }
    int kind = 0;        // 0 path_gpu, 1 volpath_gpu
    int maxDepth = 1000; // path.cpp:9, volPath.cpp:12

protected:
    // integrator.h:31-35
    void notifyUpdate(int sampleIndex, const Film& film) {
        if (m_callback && !m_stopRequested) m_callback(sampleIndex, film);
    }
    std::atomic<bool> m_stopRequested{false};
    RenderCallback m_callback;
};

// Allocator whose construct() without arguments default-initialises: resize() of an
// array of trivially constructible records reserves it without writing it, so the host
// threads that fill the array (Scene::build) are the first to touch its pages.
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind { using other = UninitAlloc<U>; };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible_v<U>) { ::new (static_cast<void*>(p)) U; }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
template <typename T>
using FlatArray = std::vector<T, UninitAlloc<T>>;

// Flattened scene: owner of the arrays a gnd_scene_desc points at. The per-triangle
// arrays are FlatArrays; Scene::build writes every element.
struct FlatScene {
    FlatArray<gnd::Node4> nodes;
    FlatArray<gnd::Tri> tris;
    FlatArray<gnd::TriAttr> attrs;
    std::vector<gnd::InstTrav> instT;
    std::vector<gnd::InstShade> instS;
    std::vector<uint32_t> tlasList;
    std::vector<gnd::Material> materials;
    std::vector<gnd::Emitter> emitters;
    std::vector<gnd::Medium> media;
    std::vector<gnd::MeshRec> meshes;
    FlatArray<float> cdf;
    FlatArray<uint32_t> origToLeaf;
    std::vector<gnd::InstMotion> motion;   // per instance when any instance moves, else empty
    std::vector<float> envTexels, envDist;
    TexTables textures;
    int envEmitter = -1, envWidth = 0, envHeight = 0;
    float envMarginalIntegral = 0.0f, envStrength = 1.0f;
    gnd::Camera camera{};
    uint32_t tlasRoot = gnd::kEmpty;
    gnd_scene_desc desc{};
    void fillDesc();
};

// scene.cpp:9-75
class Scene : public GndObject {
public:
    explicit Scene(const PropertyList&) {}
    void addChild(std::shared_ptr<GndObject> c) override;
    void activate() override;                 // builds and flattens, then integrator->preprocess
    void build();                             // builds and flattens only
    Film* ensureFilm();                       // the camera's film, created on first use
    EClassType getClassType() const override { return EScene; }
    void render() { m_integrator->render(this); }
    std::shared_ptr<CameraObj> getCamera() { return m_camera; }
    std::shared_ptr<SamplerObj> getSampler() { return m_sampler; }
    std::shared_ptr<Integrator> getIntegrator() { return m_integrator; }
    const FlatScene& flat() const { return *m_flat; }
    bool deferPreprocess = false;
    // mesh trees left to the device builder: triangles stay in their original order and
    // the flattened scene holds only the top-level tree (gnd_scene_desc.blas_on_device)
    bool deviceBlas = false;

    std::vector<std::shared_ptr<PrimitiveObj>> m_primitives;
    // emitters in the order the scene file adds them (scene.cpp:9-43): a primitive's
    // area light (prim >= 0) or a standalone emitter
    struct EmitterEntry {
        int prim;
        std::shared_ptr<EmitterObj> emitter;
    };
    std::vector<EmitterEntry> m_emitterOrder;
    std::shared_ptr<EmitterObj> m_envMap;
    std::shared_ptr<CameraObj> m_camera;
    std::shared_ptr<SamplerObj> m_sampler;
    std::shared_ptr<Integrator> m_integrator;
    std::unique_ptr<FlatScene> m_flat;
    // FileResolver::getOutputPath / getOutputName (parser.cpp:220-223): the scene file's
    // directory and stem, where the film's images are written
    std::string outputPath = ".", outputName = "output";
};

// parser.cpp:220-235
std::shared_ptr<GndObject> loadFromXML(const std::string& path, bool deferPreprocess, bool deviceBlas = false);
// mesh.cpp:148-229
void loadOBJ(const std::string& path, ShapeObj& mesh);

// ---------------------------------------------------------------- BVH build
// bvhBuilder.cpp:59-182: binary SAH tree. Returns nodes in depth-first order; leaf ranges
// index `order` (the permutation of the input primitives, leaf-contiguous).
struct BinNode {
    Bounds b;
    uint32_t offset;     // leaf: first in `order`; interior: right child index
    uint32_t count;      // 0 for interior
};
struct BinTree {
    std::vector<BinNode> nodes;
    std::vector<uint32_t> order;
};
BinTree buildSAH(const std::vector<Bounds>& primBounds, const std::vector<V3>& centroids, int parallelDepth);

// bvhBuilder.cpp:184-262 + leaf encoding: appends 4-wide nodes to `out`; leaves become
// references to [leafBase + first, +count). Returns the root node index.
uint32_t collapseToNode4(const BinTree& t, uint32_t leafBase, const std::vector<Bounds>& primBounds,
                         std::vector<gnd::Node4>& out);

}  // namespace gndh
