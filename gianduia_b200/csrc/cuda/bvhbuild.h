// Device build of the per-mesh bottom-level trees (the work of the host SAH builder,
// bvhBuilder.cpp:59-262, moved to the GPU for scene admission).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gnd/layout.h"
#include "runtime.h"

namespace gnd {

struct MeshTreeInput {
    const Node4* tlasNodes;       // host: the top-level tree (it goes first)
    uint32_t numTlasNodes;
    const uint32_t* meshBase;     // host: numMeshes + 1 prefix sums of triangles per mesh
    int numMeshes;
    const Tri* tris;              // device: original order, mesh m at meshBase[m]
    const TriAttr* attrs;         // device, same order
    int64_t numTris;
    InstTrav* instT;              // device: blasRoot of mesh instances is set
    const InstShade* instS;       // device: meshId of each instance
    int numInstances;
    uint32_t* origToLeaf;         // device, numTris entries (global original index -> slot)
    int leafMax;                  // largest leaf (1..kLeafMax)
    int numSMs;
};

struct MeshTreeOutput {
    PoolBuf nodes;                // top-level nodes, then the mesh trees
    PoolBuf tris, attrs;          // leaf order
    uint32_t numNodes = 0;
    bool nonFinite = false;       // a triangle has a NaN or infinite coordinate
    float ms = 0.0f;              // device time of the build
};

// Builds one 4-wide tree per mesh on stream `st` and waits for it.
MeshTreeOutput buildMeshTrees(const MeshTreeInput& in, cudaStream_t st);

}  // namespace gnd
