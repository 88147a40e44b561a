// Device-resident scene layout (HBM). The host builder writes these records; the
// kernels read them. All records are plain data, 16-byte aligned, sized in multiples
// of 16 bytes so they load as float4/uint4.
#pragma once
#include <cstdint>
#include "vmath.h"

namespace gnd {

// ---------------------------------------------------------------- BVH4 node
// One 4-wide node = 128 bytes = one 128-byte cache line (aligned to 128):
//   lox, hix, loy, hiy, loz, hiz : float[4] each, child i bounds (empty: +inf/-inf)
//   child[4]                     : encoded child references (see below)
//   pad[4]
// Child reference:
//   kEmpty                       : no child
//   bit31 == 0                   : inner node index
//   bit31 == 1                   : leaf; bits 27..30 = count-1 (1..16), bits 0..26 = first
//                                  (first triangle for a bottom-level tree, first entry of
//                                  the instance list for the top-level tree)
struct alignas(128) Node4 {
    float lox[4], hix[4], loy[4], hiy[4], loz[4], hiz[4];
    uint32_t child[4];
    uint32_t pad[4];
};
static_assert(sizeof(Node4) == 128, "Node4 must be 128 bytes");

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr int kLeafMax = 16;
constexpr uint32_t kLeafFirstMask = (1u << 27) - 1;

GND_HD bool isLeaf(uint32_t c) { return (c & kLeafBit) != 0; }
GND_HD uint32_t leafFirst(uint32_t c) { return c & kLeafFirstMask; }
GND_HD uint32_t leafCount(uint32_t c) { return ((c >> 27) & 15u) + 1u; }
GND_HD uint32_t makeLeaf(uint32_t first, uint32_t count) { return kLeafBit | ((count - 1u) << 27) | first; }

// ---------------------------------------------------------------- triangles
// Leaf-ordered triangle records for traversal: v0.xyz + original triangle index (bits),
// v1.xyz, v2.xyz. The edges e1 = v1 - v0, e2 = v2 - v0 are formed in the kernel exactly
// as the reference's 4-lane test forms them (mesh.cpp:264-265).
struct alignas(16) Tri {
    float v0x, v0y, v0z; uint32_t prim;
    float v1x, v1y, v1z; uint32_t pad1;
    float v2x, v2y, v2z; uint32_t pad2;
};
static_assert(sizeof(Tri) == 48, "Tri must be 48 bytes");

// Shading attributes, same leaf order as Tri: normals of the three corners and uvs.
struct alignas(16) TriAttr {
    float n0x, n0y, n0z, n1x;
    float n1y, n1z, n2x, n2y;
    float n2z, u0, v0_, u1;
    float v1_, u2, v2_, flags;   // flags: bit0 has normals, bit1 has uvs (as float)
};
static_assert(sizeof(TriAttr) == 64, "TriAttr must be 64 bytes");

// ---------------------------------------------------------------- instances
enum ShapeKind : uint32_t { kShapeMesh = 0, kShapeSphere = 1, kShapeCube = 2 };

// Traversal record (64 bytes): world-to-object 3x4 plus the shape reference.
struct alignas(16) InstTrav {
    Xf34 w2o;                 // 48 B
    uint32_t kind;            // ShapeKind
    uint32_t blasRoot;        // mesh: root node index
    float p0, p1;             // sphere: radius; cube: extents x, y (z in InstShade)
};
static_assert(sizeof(InstTrav) == 64, "InstTrav must be 64 bytes");
// InstTrav::kind flag: the instance moves (its InstMotion record holds the motion)
constexpr uint32_t kInstAnimated = 0x80000000u;

// Motion of an animated instance or camera (animated.cpp): translation, rotation
// quaternion (x, y, z, w) and scale of the start (time 0) and end (time 1) transforms,
// and the end transform's matrices (used at time >= 1; the start ones are the instance's
// or camera's own).
struct alignas(16) InstMotion {
    float t0[3]; float pad0;
    float q0[4];
    float s0[3]; float pad1;
    float t1[3]; float pad2;
    float q1[4];
    float s1[3]; float pad3;
    Xf34 endO2W;
    Xf34 endW2O;
};
static_assert(sizeof(InstMotion) == 192, "InstMotion must be 192 bytes");

// Shading record (96 bytes).
struct alignas(16) InstShade {
    Xf34 o2w;                 // 48 B object-to-world
    int32_t material;         // material index
    int32_t emitter;          // emitter index or -1
    int32_t mediumIn, mediumOut;   // material media (-1: none); only glass/index set them
    uint32_t triBase;         // first triangle (leaf order) of the mesh
    uint32_t meshId;          // mesh record index (area CDF)
    float ext[3];             // cube extents
    float radius;             // sphere radius
    uint32_t hasMedia;        // 1 when the material attaches a medium interface
    uint32_t pad;
};
static_assert(sizeof(InstShade) == 96, "InstShade must be 96 bytes");

// Mesh record for emitter sampling: its area CDF and triangles in original order.
struct alignas(16) MeshRec {
    uint32_t cdfOffset;       // into the cdf array (numTris + 1 entries)
    uint32_t numTris;
    uint32_t origToLeaf;      // offset into the original-order -> leaf-slot map
    float totalArea;
};

// ---------------------------------------------------------------- materials
enum MatType : uint32_t {
    kMatMatte = 0, kMatPlastic = 1, kMatConductor = 2, kMatGlass = 3, kMatIndex = 4
};
// Color texture slot: constant (kind 0), checkerboard (kind 1, checkerboard.h:36-48) or
// a texture tree (kind kTexNode): node `node` of SceneView::texNodes
enum : uint32_t { kTexConstant = 0, kTexChecker = 1, kTexNode = 2 };
struct alignas(16) ColorTex {
    float v1[3]; uint32_t kind;
    float v2[3]; uint32_t node;
    float scale[2], delta[2];
};
static_assert(sizeof(ColorTex) == 48, "ColorTex must be 48 bytes");

// Texture tree node: the procedural textures (textures/perlin.h, marble.h, wood.h,
// cellular.h), image textures (imageTexture.cpp) and the domain warp (domainWarp.h), with
// constant and checkerboard leaves where a warp's inputs are those.
enum TexNodeKind : int32_t {
    kTnConstant = 0, kTnChecker = 1, kTnPerlin = 2, kTnMarble = 3, kTnWood = 4, kTnCellular = 5, kTnImage = 6, kTnWarp = 7
};
enum : int32_t {
    kTnCracks = 1,              // cellular: f2 - f1 instead of f1
    kTnMetricShift = 1,         // cellular: bits 1-2 = 0 euclidean, 1 manhattan, 2 chebyshev
    kTnLinear = 1,              // image: bilinear instead of closest texel
    kTnClamp = 2,               // image: clamp instead of repeat
    kTnFloatLerp = 8,           // perlin / marble / wood float textures: std::lerp blend
    kTnNormal = 16              // image_normal: 2 c - 1 of the rgb, (0, 0, 1) below 3 channels
};
// Nesting of warps in the `warp` input of a warp: at most this many levels.
constexpr int kTexWarpNesting = 2;
// Octaves of Perlin turbulence a texture may ask for.
constexpr int kTexMaxOctaves = 64;
struct alignas(16) TexNode {
    int32_t kind;               // TexNodeKind
    int32_t octaves;            // perlin / marble / wood
    float scale;                // perlin / marble / wood / cellular: p / scale
    float strength;             // warp
    float v1[3]; float veinFreq;
    float v2[3]; float turbScale;
    float axis[3];              // marble / wood (normalised)
    int32_t flags;              // cellular / image flags above
    int32_t a, b;               // warp: base node, warp node; image: first texel, channels
    int32_t w, h;               // image size (texels are rgba floats, row 0 = bottom row)
    float cscale[2], delta[2];  // checker
};
static_assert(sizeof(TexNode) == 96, "TexNode must be 96 bytes");

// roughTex / etaTex / kTex: 0 for the constant fields, else 1 + the root node of a texture
// tree evaluated per shading point (float trees give their value in every channel).
struct alignas(16) Material {
    uint32_t type;
    float roughness;          // plastic/conductor/glass
    float eta;                // plastic/glass
    uint32_t roughTex;        // roughness tree (plastic/conductor/glass)
    ColorTex a;               // matte albedo | plastic Kd | conductor R | glass R
    ColorTex b;               // plastic Ks | glass T
    float condEta[3]; uint32_t etaTex;   // eta tree: float (plastic/glass) or color (conductor)
    float condK[3]; uint32_t kTex;       // conductor k tree
    // normal map (image_normal tree) or bump map (float tree), material.h:71-117
    uint32_t normalTex, bumpTex;
    float bumpScale;
    uint32_t pad;
};
static_assert(sizeof(Material) == 160, "Material must be 160 bytes");

// ---------------------------------------------------------------- emitters, media
// Emitter kinds: area lights on primitives (area.cpp), the delta lights point, spot and
// directional (pointlight.cpp, spotlight.cpp, directional.cpp) and the environment map
// (environment.cpp). The emitter list keeps the scene file's order (scene.cpp:9-43).
enum EmitterType : int32_t { kEmitArea = 0, kEmitPoint = 1, kEmitSpot = 2, kEmitDirectional = 3, kEmitEnv = 4 };

struct alignas(16) Emitter {
    int32_t instance;         // area: the primitive carrying the light; -1 otherwise
    int32_t type;             // EmitterType
    float cosTotal;           // spot: cos of the half width
    float cosFalloff;         // spot: cos of the angle where the falloff starts
    ColorTex radiance;        // area radiance
    float pos[3];             // point / spot position
    float strength;           // environment strength
    float dir[3];             // spot axis; directional: unit direction towards the light
    float pad1;
    float color[3];           // point / spot power, directional irradiance
    float pad2;
};
static_assert(sizeof(Emitter) == 112, "Emitter must be 112 bytes");

// Environment map for the kernels: texels (rgb, row = polar angle theta from +z, column =
// azimuth) and the piecewise-constant 2D sampling tables of distribution.cpp (marginal
// over rows, one conditional per row).
struct EnvView {
    const float* texels;
    const float* margFunc;    // height
    const float* margCdf;     // height + 1
    const float* condFunc;    // height x width
    const float* condCdf;     // height x (width + 1)
    const float* condInt;     // height
    int32_t width, height;
    float margInt, strength;
    int32_t emitter;          // index in the emitter list; -1: no environment
    int32_t pad;
};

struct alignas(16) Medium {
    float sigA[3]; float g;
    float sigS[3]; float pad0;
    float sigT[3]; float pad1;
};

// ---------------------------------------------------------------- camera
enum : int32_t { kCamPerspective = 0, kCamThinLens = 1 };

struct alignas(16) Camera {
    Xf34 toWorld;             // directions: toWorld(vector)
    int32_t width, height;
    float scale, aspect;      // tan(fov/2), width/height
    float origin[3];          // toWorld(point(0,0,0)) evaluated on the host with the
    float pad;                // homogeneous divide of transform.h:330-337
    // thin lens (thinLens.cpp:13-31); unused by the pinhole camera
    int32_t kind;             // kCamPerspective / kCamThinLens
    int32_t blades;           // aperture polygon corners; < 3: disk
    float lensRadius, focalDistance;
    float k1;                 // barrel distortion
    float caAxial, caLateral; // chromatic aberration (per colour channel)
    int32_t vignetting;       // 1: weight cos^4 of the camera-space direction
    // shutter (thinLens.cpp:80-85) and motion (camera.h:20-25)
    int32_t rollingShutter;   // 1: the sample time follows the scanline
    float scanDuration, exposureDuration;
    int32_t animated;         // 1: toWorld moves to motion.endO2W over the shutter
    InstMotion motion;
};
static_assert(sizeof(Camera) == 320, "Camera record must be 320 bytes");

// ---------------------------------------------------------------- scene view
// Device pointers of one uploaded scene, passed by value to kernels (or read from an
// array of views when several scenes share one launch).
struct SceneView {
    const Node4* nodes;
    const Tri* tris;
    const TriAttr* attrs;
    const InstTrav* instT;
    const InstShade* instS;
    const uint32_t* tlasList;     // top-level leaf entries -> instance index
    const Material* materials;
    const Emitter* emitters;
    const Medium* media;
    const MeshRec* meshes;
    const float* cdf;
    const uint32_t* origToLeaf;
    const uint8_t* instClass;     // per instance: material type, kMatIndex for null-BSDF ones
    const InstMotion* motion;     // per instance, read for instances flagged kInstAnimated
    const TexNode* texNodes;      // texture trees (ColorTex kind kTexNode)
    const float* texels;          // image texture texels, 4 floats (rgba) each
    int32_t ext;                  // 1: emitters other than area lights, an environment map,
                                  // animated instances, a thin-lens or moving camera, texture
                                  // trees (the kernels' EXT variants handle these)
    int32_t numTexNodes;
    uint32_t tlasRoot;            // kEmpty when the scene has no primitives
    int32_t numEmitters;
    int32_t numInstances;
    int32_t fastBoxes;            // 1: bounds allow the fast slab test (traverse.cuh, nodeKeysFast)
    float keyLo[3];               // ray reordering: the scene's bounds as an 8 x 8 x 8 grid,
    float keyScale[3];            // cell = (p - keyLo) * keyScale
    Camera camera;
    EnvView env;
};

}  // namespace gnd
