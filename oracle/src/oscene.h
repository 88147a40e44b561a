// Oracle (test infrastructure only): the reference's scene object model (plugin
// objects created from XML by name), BVH builder, BVH4 traversal and shapes,
// restated on the CPU. Used only as the checker for the GPU path.
#pragma once
#include "omath.h"
#include "omotion.h"
#include "osampling.h"
#include "obsdf.h"
#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- properties
// propertyList.h:12-100
struct PropertyList {
    std::map<std::string, bool> b;
    std::map<std::string, int> i;
    std::map<std::string, float> f;
    std::map<std::string, std::string> s;
    std::map<std::string, Vec3> p3, v3;
    std::map<std::string, Vec2> v2, p2;
    std::map<std::string, Color> c;
    std::map<std::string, Transform> t;
    template <typename M, typename V>
    static V get(const M& m, const std::string& k, const V& d) { auto it = m.find(k); return it == m.end() ? d : it->second; }
    bool getBoolean(const std::string& k, bool d = false) const { return get(b, k, d); }
    int getInteger(const std::string& k, int d = 0) const { return get(i, k, d); }
    float getFloat(const std::string& k, float d = 0.f) const { return get(f, k, d); }
    std::string getString(const std::string& k, const std::string& d = "") const { return get(s, k, d); }
    Vec3 getVector3(const std::string& k, const Vec3& d = Vec3()) const { return get(v3, k, d); }
    Vec2 getVector2(const std::string& k, const Vec2& d = Vec2()) const { return get(v2, k, d); }
    Vec2 getPoint2(const std::string& k, const Vec2& d = Vec2()) const { return get(p2, k, d); }
    Color getColor(const std::string& k, const Color& d = Color(0.f)) const { return get(c, k, d); }
    Transform getTransform(const std::string& k, const Transform& d = Transform()) const { return get(t, k, d); }
    bool hasColor(const std::string& k) const { return c.count(k) > 0; }
    bool hasFloat(const std::string& k) const { return f.count(k) > 0; }
    bool hasTransform(const std::string& k) const { return t.count(k) > 0; }
};

// object.h:11-23
enum ClassType { EScene, EPrimitive, EShape, ECamera, EIntegrator, ESampler, ETexture, EMaterial, EEmitter, EFilter, EMedium };
const char* classTypeName(ClassType t);

struct Object {
    std::string name;
    virtual ~Object() = default;
    virtual void addChild(std::shared_ptr<Object>) { throw std::runtime_error("addChild() not implemented!"); }
    virtual void activate() {}
    virtual ClassType classType() const = 0;
    // directory of the scene file, for objects that read files (FileResolver::resolve)
    virtual void setBaseDir(const std::string&) {}
};
using ObjectPtr = std::shared_ptr<Object>;

// factory.h:26-36, factory.cpp:17-22
std::unique_ptr<Object> createInstance(const std::string& type, const PropertyList& props);

struct Primitive;
struct Scene;
class Medium;

// shape.h:13-23
struct MediumInterface {
    const Medium* inside = nullptr;
    const Medium* outside = nullptr;
};

// shape.h:26-52
struct SurfaceInteraction {
    float t = 0.f;
    Vec3 p;
    Vec2 uv;
    float time = 0.f;
    Vec3 n;
    Vec3 dpdu;
    const Primitive* primitive = nullptr;
    uint32_t primIndex = 0;
    BSDF* bsdf = nullptr;
    MediumInterface mediumInterface;
    const Medium* getMedium(const Vec3& w) const { return Dot(w, n) > 0.0f ? mediumInterface.outside : mediumInterface.inside; }
};

// ---------------------------------------------------------------- textures
template <typename T>
struct Texture : Object {
    ClassType classType() const override { return ETexture; }
    virtual T evaluate(const SurfaceInteraction& si) const = 0;
};
using ColorTexture = Texture<Color>;
using FloatTexture = Texture<float>;

// ---------------------------------------------------------------- BVH
// bvhBuilder.h:8-19
struct BVHNode {
    Bounds3 bounds;
    uint32_t offset = 0;   // leaf: first primitive; interior: right child index
    uint16_t nPrimitives = 0;
    uint8_t axis = 0;
};
// bvhBuilder.h:21-28
struct alignas(16) BVHNode4 {
    float minX[4], minY[4], minZ[4];
    float maxX[4], maxY[4], maxZ[4];
    uint32_t offset[4];
    uint32_t packCount[4];
    uint8_t childType[4];   // 0 empty, 1 inner, 2 leaf
};
// bvhBuilder.h:30-39
struct BVHBuildInfo { Bounds3 bounds; Vec3 centroid; int originalIndex; };
struct BVHBuildResult { std::vector<BVHNode> nodes; std::vector<int> orderedIndices; };
// bvhBuilder.cpp:59-262
BVHBuildResult buildBVH(std::vector<BVHBuildInfo>& data);
std::vector<BVHNode4> buildWide(const std::vector<BVHNode>& bin);

// Traversal counters (not in the reference): per-ray node visits and triangle tests,
// used as the implementation-independent work measure for the GPU roofline.
struct TraversalStats { uint64_t nodes = 0, tris = 0, leaves = 0; };

// bvhTraversal.h:19-98. visit(offset, count) returns true on a hit; tMax is re-read.
bool traverseBVH4(const std::vector<BVHNode4>& nodes, const Ray& ray, bool shadow,
                  const std::function<bool(int, int)>& leaf, TraversalStats* st);

// ---------------------------------------------------------------- shapes
struct Shape : Object {
    ClassType classType() const override { return EShape; }
    virtual bool rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats* st) const = 0;
    virtual void fillInteraction(const Ray& ray, SurfaceInteraction& si) const = 0;
    virtual Bounds3 getBounds() const = 0;
    virtual float sampleSurface(const Vec3& ref, const Vec2& u, SurfaceInteraction& info) const = 0;
    virtual float pdfSurface(const Vec3& ref, const SurfaceInteraction& info) const = 0;
};

// mesh.h:37-44
struct TrianglePack4 {
    float v0x[4], v0y[4], v0z[4];
    float v1x[4], v1y[4], v1z[4];
    float v2x[4], v2y[4], v2z[4];
    uint32_t primIndex[4];
};

struct Mesh : Shape {
    std::string filename;
    std::vector<Vec3> positions, normals;
    std::vector<Vec2> uvs;
    std::vector<uint32_t> indices;
    std::vector<TrianglePack4> packs;
    std::vector<BVHNode4> nodes4;
    Bounds3 bounds;
    std::vector<float> cdf;
    float totalArea = 0.f;
    explicit Mesh(const PropertyList& p) : filename(p.getString("filename", "")) {}
    void activate() override;           // mesh.cpp:17-146
    void loadOBJ(const std::string& f); // mesh.cpp:148-229
    void buildAccel();                  // mesh.cpp:29-146 (after geometry is present)
    bool rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats* st) const override;
    void fillInteraction(const Ray& ray, SurfaceInteraction& si) const override;
    Bounds3 getBounds() const override { return bounds; }
    float sampleSurface(const Vec3& ref, const Vec2& u, SurfaceInteraction& info) const override;
    float pdfSurface(const Vec3&, const SurfaceInteraction&) const override { return totalArea > 0.f ? 1.0f / totalArea : 0.f; }
};

struct Sphere : Shape {
    float radius;
    explicit Sphere(const PropertyList& p) : radius(p.getFloat("radius", 1.0f)) {}
    bool rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats* st) const override;
    void fillInteraction(const Ray& ray, SurfaceInteraction& si) const override;
    Bounds3 getBounds() const override { return Bounds3(Vec3(-radius), Vec3(radius)); }
    float sampleSurface(const Vec3& ref, const Vec2& u, SurfaceInteraction& info) const override;
    float pdfSurface(const Vec3&, const SurfaceInteraction&) const override { return Inv4Pi / (radius * radius); }
};

struct Cube : Shape {
    Vec3 ext, mn, mx;
    explicit Cube(const PropertyList& p) : ext(p.getVector3("extents", Vec3(1.0f))), mn(-ext.x, -ext.y, -ext.z), mx(ext) {}
    bool rayIntersect(const Ray& ray, SurfaceInteraction& si, bool predicate, TraversalStats* st) const override;
    void fillInteraction(const Ray& ray, SurfaceInteraction& si) const override;
    Bounds3 getBounds() const override { return Bounds3(mn, mx); }
    float sampleSurface(const Vec3& ref, const Vec2& u, SurfaceInteraction& info) const override;
    float pdfSurface(const Vec3&, const SurfaceInteraction&) const override {
        Vec3 d = mx - mn;
        return 1.0f / (2.0f * (d.x * d.y + d.x * d.z + d.y * d.z));
    }
};

// ---------------------------------------------------------------- media
// medium.h:13-25
struct MediumInteraction {
    Vec3 p, wo;
    const Medium* medium = nullptr;
    Color sigma_a, sigma_s;
    const HGPhase* phase = nullptr;
    bool isValid() const { return medium != nullptr; }
};
class Medium : public Object {
public:
    ClassType classType() const override { return EMedium; }
    virtual Color Tr(const Ray& ray) const = 0;
    virtual Color sample(const Ray& ray, Sampler& s, Arena& a, MediumInteraction& mi) const = 0;
};
// homogeneous.cpp:14-63
class HomogeneousMedium : public Medium {
public:
    Color sigma_a, sigma_s, sigma_t;
    float g;
    explicit HomogeneousMedium(const PropertyList& p);
    Color Tr(const Ray& ray) const override;
    Color sample(const Ray& ray, Sampler& s, Arena& a, MediumInteraction& mi) const override;
    Color sampleU(const Ray& ray, float u0, float u1, Arena& a, MediumInteraction& mi) const;
};

// ---------------------------------------------------------------- materials
struct Material : Object {
    std::shared_ptr<Medium> inside, outside;
    std::shared_ptr<Texture<Color>> normalMap;   // image_normal: (x, y, z) in r, g, b
    std::shared_ptr<Texture<float>> bumpMap;
    float bumpScale = 1.0f;                      // material.h:14
    ClassType classType() const override { return EMaterial; }
    void addChild(ObjectPtr child) override;   // material.h:36-59
    virtual void computeScatteringFunctions(SurfaceInteraction& si, Arena& a) const = 0;
    void applyNormalOrBump(SurfaceInteraction& si) const;   // material.h:71-117
    // material.h:119-126
    void applyMediums(SurfaceInteraction& si) const {
        if (inside || outside) si.mediumInterface = MediumInterface{inside.get(), outside.get()};
    }
};

// ---------------------------------------------------------------- emitters
struct Emitter : Object {
    const Primitive* prim = nullptr;
    ClassType classType() const override { return EEmitter; }
    virtual Color eval(const SurfaceInteraction& si, const Vec3& w) const = 0;
    virtual Color sample(const SurfaceInteraction& ref, const Vec2& u, SurfaceInteraction& info, float& pdf, Ray& shadowRay) const = 0;
    virtual float pdf(const SurfaceInteraction& ref, const SurfaceInteraction& info) const = 0;
    virtual bool isDelta() const { return false; }             // emitter.h: EMITTER_DELTA
    virtual bool isInfiniteAreaLight() const { return false; }  // environment.cpp:93
};

// ---------------------------------------------------------------- primitive
// primitive.cpp:7-76 (static transforms only)
struct Primitive : Object {
    std::shared_ptr<Shape> shape;
    std::shared_ptr<Material> material;
    std::shared_ptr<Emitter> emitter;
    Transform toWorld;            // the start transform
    AnimatedTransform anim;       // toWorld -> toWorldEnd over time [0, 1]
    int originalIndex = -1;
    explicit Primitive(const PropertyList& p);
    ClassType classType() const override { return EPrimitive; }
    void addChild(ObjectPtr child) override;
    void activate() override;
    bool rayIntersect(const Ray& rWorld, SurfaceInteraction& si, bool predicate, TraversalStats* st) const;
    void fillInteraction(const Ray& rWorld, SurfaceInteraction& si) const;
    Bounds3 getWorldBounds() const { return anim.motionBounds(shape->getBounds()); }   // primitive.cpp:74-76
    Transform getToWorld(float time) const { return anim.interpolate(time); }
};

// ---------------------------------------------------------------- camera, film
struct Filter : Object {
    Vec2 radius;
    ClassType classType() const override { return EFilter; }
    virtual float evaluate(const Vec2& p) const = 0;
};

// film.h:21-136 plus a per-pixel sum of squares (not in the reference) for
// standard errors in the statistical parity tests.
//
// Fixed-point mode (not in the reference): sum wL and sum w are accumulated as 64-bit
// integers in units of 2^-24, each term clamped to [0, 1e11] and rounded to nearest even
// before it is added -- the film the GPU keeps. Integer sums do not depend on the order of
// the additions, so renders of disjoint pass ranges add up to one render of all of them
// bit for bit (the multi-rank reduction checks this).
struct Film {
    int width, height;
    std::shared_ptr<Filter> filter;
    std::vector<std::atomic<float>> sum;   // 7 floats per pixel: wL(3), w, wL^2(3)
    bool fixedMode = false;
    std::vector<std::atomic<uint64_t>> fixedSum;   // fixedMode: 4 per pixel: wL(3), w
    Film(int w, int h, std::shared_ptr<Filter> f);
    void enableFixed();
    void addSample(const Vec2& pFilm, const Color& L);
    void clear();
};
// One term of the fixed-point film: clamp to [0, 1e11], scale by 2^24, round to nearest even.
uint64_t toFixed(float x);

// camera.h CameraSample
struct CameraSample {
    Vec2 pFilm, pLens;
    float lambdaOffset = 0.0f, time = 0.0f;
};

struct Camera : Object {
    Transform toWorld;
    AnimatedTransform anim;   // toWorld -> toWorldEnd over the shutter time [0, 1]
    int width, height;
    float fov, scale;
    // thinLens.cpp:13-31 (kind 1); kind 0 is the pinhole `perspective` camera
    int kind = 0;
    float lensRadius = 0.0f, focalDistance = 10.0f, k1 = 0.0f, caAxial = 0.0f, caLateral = 0.0f;
    bool vignetting = false, rollingShutter = false;
    int blades = 0;
    float scanDuration = 0.9f, exposureDuration = 0.1f;
    std::shared_ptr<Filter> filterObj;
    Camera(const PropertyList& p, int kind);
    ClassType classType() const override { return ECamera; }
    void addChild(ObjectPtr child) override;
    float aspect() const { return width / (float)height; }
    bool hasChromaticAberration() const { return kind == 1 && (caLateral != 0.0f || caAxial != 0.0f); }
    // perspective.cpp:15-32 / thinLens.cpp:33-91; returns the ray weight
    float shootRay(const CameraSample& s, Ray* ray) const;
};

struct SamplerObj : Object {
    int spp;
    explicit SamplerObj(const PropertyList& p) : spp(p.getInteger("spp", 1)) {}
    ClassType classType() const override { return ESampler; }
};

struct IntegratorObj : Object {
    int kind;   // 0 path, 1 volpath
    int maxDepth;
    IntegratorObj(int k, const PropertyList& p) : kind(k), maxDepth(p.getInteger("maxDepth", 1000)) {}
    ClassType classType() const override { return EIntegrator; }
};

// ---------------------------------------------------------------- scene
// scene.cpp:9-71, bvh.cpp:10-66
struct Scene : Object {
    std::vector<std::shared_ptr<Primitive>> prims;   // reordered by the TLAS build
    std::vector<std::shared_ptr<Emitter>> emitters;  // scene-file order (scene.cpp:9-43)
    std::shared_ptr<Emitter> envMap;
    std::shared_ptr<Camera> camera;
    std::shared_ptr<SamplerObj> sampler;
    std::shared_ptr<IntegratorObj> integrator;
    std::vector<BVHNode4> nodes4;
    Bounds3 bounds;
    explicit Scene(const PropertyList&) {}
    ClassType classType() const override { return EScene; }
    void addChild(ObjectPtr child) override;
    void activate() override;
    void buildTLAS();
    bool rayIntersect(const Ray& ray, SurfaceInteraction& si, TraversalStats* st = nullptr) const;
    bool occluded(const Ray& ray, TraversalStats* st = nullptr) const;
    const Emitter* randomEmitter(float rnd) const {
        size_t n = emitters.size();
        size_t idx = std::min((size_t)std::floor(n * rnd), n - 1);
        return emitters[idx].get();
    }
};

std::shared_ptr<Object> loadSceneXML(const std::string& path);

}  // namespace orc
