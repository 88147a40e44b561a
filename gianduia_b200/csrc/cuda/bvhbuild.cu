// Device build of the per-mesh bottom-level trees, for scene admission without the host
// SAH build (bvhBuilder.cpp:59-262). All meshes of a scene are built together:
//
//   1. kPrep: per triangle its centroid (centre of its bounds); per mesh the bounds of
//      the centroids (ordered-integer atomics, warp-aggregated).
//   2. kMorton: 64-bit key = mesh index above a 3D Morton code of the centroid quantised
//      in its mesh's centroid bounds; one radix sort of (key, triangle) orders every mesh
//      by its Morton curve, meshes one after another.
//   3. kBinary: the binary radix tree of each mesh's sorted keys, built bottom-up in one
//      pass (Apetrei, "Fast and Simple Agglomerative LBVH Construction", 2014): every
//      triangle walks up from its leaf; at each internal node the first arriving child
//      records itself and stops, the second combines both and carries on. A node's
//      parent is the neighbouring split with the lower highest differing bit (equal keys
//      are told apart by their index bits). On the way up each node gets its bounds,
//      triangle count and surface-area cost, min(count * area as one leaf,
//      area + cost(left) + cost(right)), the same unit costs as the reference's SAH
//      (bvhBuilder.cpp:120-131); a subtree of at most `leafMax` triangles that is cheaper
//      as a leaf becomes one. No thread waits on another.
//   4. kRoots / kCollapse: top-down collapse to 4-wide nodes, one level per launch: a
//      node takes its binary node's two children and, like the host collapse
//      (bvhBuilder.cpp:184-262), opens the largest-area inner child until it has four;
//      leaves become leaf references (their triangles are contiguous in sorted order),
//      inner children get new nodes (allocated together) and go to the next level.
//   5. kGather / kPatch: triangles and attributes in leaf (sorted) order, the original ->
//      leaf map, and the tree root of each mesh instance.
//
// Node indices: the host's top-level nodes first, then mesh m's root at numTlasNodes + m,
// then the inner nodes level by level.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <string>

#include "bvhbuild.h"

namespace gnd {

namespace {

constexpr int kBuildBlock = 256;
constexpr uint32_t kSlotLeaf = 0x80000000u;   // in Slot::count: a leaf (one triangle or a collapsed subtree)
constexpr uint32_t kFlagNonFinite = 1u, kFlagOverflow = 2u;

// One child of a binary node, as its parent stores it: bounds, SAH cost, triangle count
// (| kSlotLeaf), the child's global internal node index and the first triangle slot of
// its range.
struct alignas(16) Slot {
    float lx, ly, lz, cost;
    float hx, hy, hz;
    uint32_t count;
    uint32_t ref, first, pad0, pad1;
};
static_assert(sizeof(Slot) == 48, "Slot must be 48 bytes");

struct QEntry {
    uint32_t node;   // mesh-tree node index (relative to the first mesh-tree node)
    uint32_t bin;    // global index of the binary internal node it expands
};

// Float <-> unsigned integer with the same order (atomicMin/atomicMax on floats).
__device__ __forceinline__ uint32_t orderedBits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fromOrderedBits(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Mesh of triangle t: the last m with base[m] <= t (empty meshes share their base with
// the next one).
__device__ __forceinline__ int meshOf(const uint32_t* base, int M, uint32_t t) {
    int lo = 0, hi = M - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(base + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct Box {
    float lx, ly, lz, hx, hy, hz;
};
__device__ __forceinline__ Box triBox(const Tri& t) {
    Box b;
    b.lx = fminf(fminf(t.v0x, t.v1x), t.v2x);
    b.ly = fminf(fminf(t.v0y, t.v1y), t.v2y);
    b.lz = fminf(fminf(t.v0z, t.v1z), t.v2z);
    b.hx = fmaxf(fmaxf(t.v0x, t.v1x), t.v2x);
    b.hy = fmaxf(fmaxf(t.v0y, t.v1y), t.v2y);
    b.hz = fmaxf(fmaxf(t.v0z, t.v1z), t.v2z);
    return b;
}
__device__ __forceinline__ bool triFinite(const Tri& t) {
    return isfinite(t.v0x) && isfinite(t.v0y) && isfinite(t.v0z) && isfinite(t.v1x) && isfinite(t.v1y) &&
           isfinite(t.v1z) && isfinite(t.v2x) && isfinite(t.v2y) && isfinite(t.v2z);
}
__device__ __forceinline__ float boxArea(float dx, float dy, float dz) {
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
__device__ __forceinline__ float slotArea(const Slot& s) {
    return boxArea(s.hx - s.lx, s.hy - s.ly, s.hz - s.lz);
}

// 21-bit value -> every third bit of a 63-bit word (bit i -> bit 3i).
__device__ __forceinline__ uint64_t spreadBits3(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// 1. centroid bounds per mesh (cb: lo xyz for every mesh, then hi xyz)
__global__ void __launch_bounds__(kBuildBlock) kPrep(const Tri* __restrict__ tris, uint32_t N,
                                                     const uint32_t* __restrict__ base, int M,
                                                     uint32_t* cbLo, uint32_t* cbHi, uint32_t* flags) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < N;
    int m = 0;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    bool finite = true;
    if (active) {
        const Tri tr = tris[t];
        finite = triFinite(tr);
        const Box b = triBox(tr);
        cx = (b.lx + b.hx) * 0.5f;
        cy = (b.ly + b.hy) * 0.5f;
        cz = (b.lz + b.hz) * 0.5f;
        m = meshOf(base, M, t);
        if (!finite) atomicOr(flags, kFlagNonFinite);
    }
    const bool use = active && finite;
    const uint32_t act = __ballot_sync(0xffffffffu, use);
    if (!act) return;
    const int leader = __ffs(act) - 1;
    const int m0 = __shfl_sync(0xffffffffu, m, leader);
    if (__all_sync(0xffffffffu, !use || m == m0)) {
        float lx = use ? cx : INFINITY, ly = use ? cy : INFINITY, lz = use ? cz : INFINITY;
        float hx = use ? cx : -INFINITY, hy = use ? cy : -INFINITY, hz = use ? cz : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) {
            lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
            ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
            lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
            hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
            hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
            hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
        }
        if ((int)(threadIdx.x & 31) == leader) {
            atomicMin(cbLo + 3 * m0 + 0, orderedBits(lx));
            atomicMin(cbLo + 3 * m0 + 1, orderedBits(ly));
            atomicMin(cbLo + 3 * m0 + 2, orderedBits(lz));
            atomicMax(cbHi + 3 * m0 + 0, orderedBits(hx));
            atomicMax(cbHi + 3 * m0 + 1, orderedBits(hy));
            atomicMax(cbHi + 3 * m0 + 2, orderedBits(hz));
        }
    } else if (use) {
        atomicMin(cbLo + 3 * m + 0, orderedBits(cx));
        atomicMin(cbLo + 3 * m + 1, orderedBits(cy));
        atomicMin(cbLo + 3 * m + 2, orderedBits(cz));
        atomicMax(cbHi + 3 * m + 0, orderedBits(cx));
        atomicMax(cbHi + 3 * m + 1, orderedBits(cy));
        atomicMax(cbHi + 3 * m + 2, orderedBits(cz));
    }
}

// 2. sort keys: mesh index above the Morton code (3 * bits bits) of the centroid
__device__ __forceinline__ uint32_t quantise(float c, float lo, float hi, float cells) {
    const float ext = hi - lo;
    const float s = ext > 0.0f ? cells / ext : 0.0f;   // NaN / empty bounds: 0
    const float q = fminf(fmaxf((c - lo) * s, 0.0f), cells - 1.0f);   // NaN -> 0
    return (uint32_t)q;
}
__global__ void __launch_bounds__(kBuildBlock) kMorton(const Tri* __restrict__ tris, uint32_t N,
                                                       const uint32_t* __restrict__ base, int M,
                                                       const uint32_t* __restrict__ cbLo, const uint32_t* __restrict__ cbHi,
                                                       int bits, uint64_t* keys, uint32_t* vals) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const int m = meshOf(base, M, t);
    const Box b = triBox(tris[t]);
    const float cells = (float)(1u << bits);
    const uint32_t qx = quantise((b.lx + b.hx) * 0.5f, fromOrderedBits(cbLo[3 * m + 0]), fromOrderedBits(cbHi[3 * m + 0]), cells);
    const uint32_t qy = quantise((b.ly + b.hy) * 0.5f, fromOrderedBits(cbLo[3 * m + 1]), fromOrderedBits(cbHi[3 * m + 1]), cells);
    const uint32_t qz = quantise((b.lz + b.hz) * 0.5f, fromOrderedBits(cbLo[3 * m + 2]), fromOrderedBits(cbHi[3 * m + 2]), cells);
    const uint64_t code = (spreadBits3(qx) << 2) | (spreadBits3(qy) << 1) | spreadBits3(qz);
    keys[t] = ((uint64_t)m << (3 * bits)) | code;
    vals[t] = t;
}

// Highest differing bit between sorted keys i and i + 1 of a mesh, keys first, then the
// local indices (so that equal keys still split): a larger rank splits nearer the root.
__device__ __forceinline__ int splitRank(const uint64_t* __restrict__ keys, uint32_t base, uint32_t i) {
    const uint64_t x = __ldg(keys + base + i) ^ __ldg(keys + base + i + 1);
    return x ? 32 + 63 - __clzll((long long)x) : 31 - __clz((int)(i ^ (i + 1u)));
}

__device__ __forceinline__ Slot loadSlotL2(const Slot* p) {
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldcg(reinterpret_cast<const float4*>(p) + 1);
    const uint4 c = __ldcg(reinterpret_cast<const uint4*>(p) + 2);
    Slot s;
    s.lx = a.x; s.ly = a.y; s.lz = a.z; s.cost = a.w;
    s.hx = b.x; s.hy = b.y; s.hz = b.z; s.count = __float_as_uint(b.w);
    s.ref = c.x; s.first = c.y; s.pad0 = c.z; s.pad1 = c.w;
    return s;
}

// 3. binary trees, bottom-up; slots[2g], slots[2g + 1]: children of internal node g
__global__ void __launch_bounds__(kBuildBlock) kBinary(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                                       const Tri* __restrict__ tris, const uint32_t* __restrict__ base,
                                                       int mortonBits, uint32_t N, Slot* slots, int* other,
                                                       Slot* rootSlot, uint32_t* innerCount, int leafMax) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int m = (int)(__ldg(keys + s) >> mortonBits);
    const uint32_t b0 = __ldg(base + m);
    const uint32_t n = __ldg(base + m + 1) - b0;
    const uint32_t i = s - b0;
    const Box tb = triBox(tris[__ldg(vals + s)]);
    Slot cur;
    cur.lx = tb.lx; cur.ly = tb.ly; cur.lz = tb.lz;
    cur.hx = tb.hx; cur.hy = tb.hy; cur.hz = tb.hz;
    cur.cost = boxArea(tb.hx - tb.lx, tb.hy - tb.ly, tb.hz - tb.lz);
    cur.count = 1u | kSlotLeaf;
    cur.ref = 0;
    cur.first = s;
    cur.pad0 = cur.pad1 = 0;
    uint32_t l = i, r = i;
    for (;;) {
        if (l == 0 && r == n - 1) {
            rootSlot[m] = cur;
            return;
        }
        const bool isLeft = (l == 0) || (r != n - 1 && splitRank(keys, b0, r) < splitRank(keys, b0, l - 1));
        const uint32_t p = isLeft ? r : l - 1;
        const uint32_t g = b0 + p;
        slots[2 * g + (isLeft ? 0 : 1)] = cur;
        __threadfence();
        const int prev = atomicExch(other + g, (int)(isLeft ? l : r));
        if (prev < 0) return;   // the sibling has not arrived: it completes the node
        __threadfence();
        const Slot sib = loadSlotL2(slots + 2 * g + (isLeft ? 1 : 0));
        if (isLeft) r = (uint32_t)prev;
        else l = (uint32_t)prev;
        Slot up;
        up.lx = fminf(cur.lx, sib.lx); up.ly = fminf(cur.ly, sib.ly); up.lz = fminf(cur.lz, sib.lz);
        up.hx = fmaxf(cur.hx, sib.hx); up.hy = fmaxf(cur.hy, sib.hy); up.hz = fmaxf(cur.hz, sib.hz);
        const uint32_t count = (cur.count & ~kSlotLeaf) + (sib.count & ~kSlotLeaf);
        const float area = boxArea(up.hx - up.lx, up.hy - up.ly, up.hz - up.lz);
        const float innerCost = area + cur.cost + sib.cost;
        const float leafCost = (float)count * area;
        const bool asLeaf = (int)count <= leafMax && leafCost <= innerCost;
        if (!asLeaf) atomicAdd(innerCount, 1u);
        up.cost = asLeaf ? leafCost : innerCost;
        up.count = count | (asLeaf ? kSlotLeaf : 0u);
        up.ref = g;
        up.first = b0 + l;
        up.pad0 = up.pad1 = 0;
        cur = up;
    }
}

__device__ __forceinline__ void setChild(Node4& nd, int k, const Slot& s, uint32_t ref) {
    nd.lox[k] = s.lx; nd.loy[k] = s.ly; nd.loz[k] = s.lz;
    nd.hix[k] = s.hx; nd.hiy[k] = s.hy; nd.hiz[k] = s.hz;
    nd.child[k] = ref;
}
__device__ __forceinline__ void clearChildren(Node4& nd, int from) {
    for (int k = from; k < 4; ++k) {
        nd.lox[k] = nd.loy[k] = nd.loz[k] = INFINITY;
        nd.hix[k] = nd.hiy[k] = nd.hiz[k] = -INFINITY;
        nd.child[k] = kEmpty;
    }
    for (int k = 0; k < 4; ++k) nd.pad[k] = 0;
}

// 4a. mesh roots: empty meshes get an empty node, a mesh that is one leaf a node with
// that leaf; the others start the collapse queue.
__global__ void kRoots(const uint32_t* __restrict__ base, int M, const Slot* __restrict__ rootSlot, Node4* nodes,
                       QEntry* queue, uint32_t* queueCount) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const uint32_t n = base[m + 1] - base[m];
    Node4 nd;
    if (n == 0) {
        clearChildren(nd, 0);
        nodes[m] = nd;
        return;
    }
    const Slot r = rootSlot[m];
    if (r.count & kSlotLeaf) {
        setChild(nd, 0, r, makeLeaf(r.first, r.count & ~kSlotLeaf));
        clearChildren(nd, 1);
        nodes[m] = nd;
        return;
    }
    const uint32_t q = atomicAdd(queueCount, 1u);
    queue[q] = QEntry{(uint32_t)m, r.ref};
}

// 4b. one level of the collapse
__global__ void __launch_bounds__(kBuildBlock) kCollapse(const QEntry* __restrict__ qin, const uint32_t* __restrict__ qinCount,
                                                         QEntry* qout, uint32_t* qoutCount, const Slot* __restrict__ slots,
                                                         Node4* nodes, uint32_t firstNode, uint32_t* nodeCount,
                                                         uint32_t capacity, uint32_t* flags) {
    const uint32_t n = *qinCount;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const QEntry e = qin[k];
        Slot c[4];
        int nc = 2;
        c[0] = slots[2 * e.bin];
        c[1] = slots[2 * e.bin + 1];
        while (nc < 4) {
            int best = -1;
            float bestArea = -1.0f;
            for (int j = 0; j < nc; ++j) {
                if (c[j].count & kSlotLeaf) continue;
                const float a = slotArea(c[j]);
                if (a > bestArea) { bestArea = a; best = j; }
            }
            if (best < 0) break;
            const uint32_t b = c[best].ref;
            c[best] = slots[2 * b];
            c[nc++] = slots[2 * b + 1];
        }
        uint32_t inner = 0;
        for (int j = 0; j < nc; ++j) inner += (c[j].count & kSlotLeaf) ? 0u : 1u;
        uint32_t first = 0, q = 0;
        if (inner) {
            first = atomicAdd(nodeCount, inner);
            q = atomicAdd(qoutCount, inner);
            if (first + inner > capacity || q + inner > capacity) {
                atomicOr(flags, kFlagOverflow);
                continue;
            }
        }
        Node4 nd;
        uint32_t k2 = 0;
        for (int j = 0; j < nc; ++j) {
            if (c[j].count & kSlotLeaf) {
                setChild(nd, j, c[j], makeLeaf(c[j].first, c[j].count & ~kSlotLeaf));
            } else {
                setChild(nd, j, c[j], firstNode + first + k2);
                qout[q + k2] = QEntry{first + k2, c[j].ref};
                ++k2;
            }
        }
        clearChildren(nd, nc);
        nodes[e.node] = nd;
    }
}

// 5. leaf-ordered triangles and attributes, original -> leaf map, instance roots
__global__ void __launch_bounds__(kBuildBlock) kGather(const uint32_t* __restrict__ vals, uint32_t N,
                                                       const Tri* __restrict__ tris, const TriAttr* __restrict__ attrs,
                                                       Tri* trisOut, TriAttr* attrsOut, uint32_t* origToLeaf) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t o = vals[s];
    trisOut[s] = tris[o];
    attrsOut[s] = attrs[o];
    origToLeaf[o] = s;
}

__global__ void kPatch(InstTrav* instT, const InstShade* __restrict__ instS, int numInstances,
                       const uint32_t* __restrict__ base, int M, uint32_t firstNode) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numInstances || (instT[i].kind & ~kInstAnimated) != kShapeMesh) return;
    const uint32_t m = instS[i].meshId;
    instT[i].blasRoot = ((int)m < M && base[m + 1] > base[m]) ? firstNode + m : kEmpty;
}

inline unsigned blocksFor(uint64_t n) { return (unsigned)((n + kBuildBlock - 1) / kBuildBlock); }

}  // namespace

MeshTreeOutput buildMeshTrees(const MeshTreeInput& in, cudaStream_t st) {
    MeshTreeOutput out;
    const int M = in.numMeshes;
    if (M < 0 || in.numTris < 0 || in.numTris >= (int64_t)kLeafFirstMask) throw Error(GND_ERR_INVALID, "mesh tree build: bad sizes");
    if (in.leafMax < 1 || in.leafMax > kLeafMax) throw Error(GND_ERR_INVALID, "mesh tree build: leaf size out of range");
    const uint32_t N = (uint32_t)in.numTris;
    if (M > 0) {
        if (in.meshBase[0] != 0 || in.meshBase[M] != N) throw Error(GND_ERR_INVALID, "mesh tree build: mesh ranges do not cover the triangles");
        for (int m = 0; m < M; ++m)
            if (in.meshBase[m + 1] < in.meshBase[m]) throw Error(GND_ERR_INVALID, "mesh tree build: mesh ranges out of order");
    } else if (N != 0) {
        throw Error(GND_ERR_INVALID, "mesh tree build: triangles without meshes");
    }
    const uint32_t T = in.numTlasNodes;
    cudaEvent_t e0, e1;
    GND_CUDA(cudaEventCreate(&e0));
    GND_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evg{e0, e1};
    GND_CUDA(cudaEventRecord(e0, st));

    PoolBuf base((size_t)(M + 1) * 4, st);
    if (M > 0) GND_CUDA(cudaMemcpyAsync(base.ptr, in.meshBase, (size_t)(M + 1) * 4, cudaMemcpyHostToDevice, st));
    PoolBuf flags(16, st), counters(16, st);
    GND_CUDA(cudaMemsetAsync(flags.ptr, 0, 16, st));
    GND_CUDA(cudaMemsetAsync(counters.ptr, 0, 16, st));
    uint32_t* innerCount = counters.as<uint32_t>();
    uint32_t* nodeCount = counters.as<uint32_t>() + 1;

    PoolBuf blas, keysB, valsB;
    uint32_t numBlas = 0;
    if (N > 0) {
        // 1-2. centroid bounds and keys
        PoolBuf cb((size_t)M * 24, st);
        uint32_t* cbLo = cb.as<uint32_t>();
        uint32_t* cbHi = cbLo + 3 * (size_t)M;
        GND_CUDA(cudaMemsetAsync(cbLo, 0xff, (size_t)M * 12, st));
        GND_CUDA(cudaMemsetAsync(cbHi, 0x00, (size_t)M * 12, st));
        kPrep<<<blocksFor(N), kBuildBlock, 0, st>>>(in.tris, N, base.as<uint32_t>(), M, cbLo, cbHi, flags.as<uint32_t>());
        GND_CUDA(cudaGetLastError());
        const int meshBits = M > 1 ? 32 - __builtin_clz((unsigned)(M - 1)) : 0;
        const int bits = std::min(21, (63 - meshBits) / 3);
        const int endBit = 3 * bits + meshBits;
        PoolBuf keysA((size_t)N * 8, st), valsA((size_t)N * 4, st);
        keysB = PoolBuf((size_t)N * 8, st);
        valsB = PoolBuf((size_t)N * 4, st);
        kMorton<<<blocksFor(N), kBuildBlock, 0, st>>>(in.tris, N, base.as<uint32_t>(), M, cbLo, cbHi, bits,
                                                       keysA.as<uint64_t>(), valsA.as<uint32_t>());
        GND_CUDA(cudaGetLastError());
        size_t tempBytes = 0;
        GND_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keysA.as<uint64_t>(), keysB.as<uint64_t>(),
                                                 valsA.as<uint32_t>(), valsB.as<uint32_t>(), (int)N, 0, endBit, st));
        PoolBuf temp(std::max<size_t>(tempBytes, 16), st);
        GND_CUDA(cub::DeviceRadixSort::SortPairs(temp.ptr, tempBytes, keysA.as<uint64_t>(), keysB.as<uint64_t>(),
                                                 valsA.as<uint32_t>(), valsB.as<uint32_t>(), (int)N, 0, endBit, st));
        // 3. binary trees
        PoolBuf slots((size_t)N * 2 * sizeof(Slot), st), other((size_t)N * 4, st), roots((size_t)M * sizeof(Slot), st);
        GND_CUDA(cudaMemsetAsync(other.ptr, 0xff, (size_t)N * 4, st));
        kBinary<<<blocksFor(N), kBuildBlock, 0, st>>>(keysB.as<uint64_t>(), valsB.as<uint32_t>(), in.tris, base.as<uint32_t>(),
                                                       3 * bits, N, slots.as<Slot>(), other.as<int>(), roots.as<Slot>(),
                                                       innerCount, in.leafMax);
        GND_CUDA(cudaGetLastError());
        uint32_t inner = 0;
        GND_CUDA(cudaMemcpyAsync(&inner, innerCount, 4, cudaMemcpyDeviceToHost, st));
        GND_CUDA(cudaStreamSynchronize(st));
        // 4. collapse: at most one node per inner binary node, plus the mesh roots
        const uint32_t capacity = inner + (uint32_t)M;
        blas = PoolBuf((size_t)capacity * sizeof(Node4), st);
        PoolBuf qa((size_t)capacity * sizeof(QEntry), st), qb((size_t)capacity * sizeof(QEntry), st), qcount(16, st);
        uint32_t* qc = qcount.as<uint32_t>();
        GND_CUDA(cudaMemsetAsync(qc, 0, 16, st));
        const uint32_t first = (uint32_t)M;
        GND_CUDA(cudaMemcpyAsync(nodeCount, &first, 4, cudaMemcpyHostToDevice, st));
        kRoots<<<blocksFor((uint64_t)M), kBuildBlock, 0, st>>>(base.as<uint32_t>(), M, roots.as<Slot>(), blas.as<Node4>(),
                                                                qa.as<QEntry>(), qc);
        GND_CUDA(cudaGetLastError());
        const unsigned grid = std::max(1u, std::min(blocksFor(capacity), (unsigned)(in.numSMs * 8)));
        QEntry* cur = qa.as<QEntry>();
        QEntry* nxt = qb.as<QEntry>();
        int c = 0;
        for (int level = 0;; ++level) {
            if (level > 1024) throw Error(GND_ERR_DEVICE_CHECK, "mesh tree build: collapse did not finish");
            GND_CUDA(cudaMemsetAsync(qc + (c ^ 1), 0, 4, st));
            kCollapse<<<grid, kBuildBlock, 0, st>>>(cur, qc + c, nxt, qc + (c ^ 1), slots.as<Slot>(), blas.as<Node4>(),
                                                     T, nodeCount, capacity, flags.as<uint32_t>());
            GND_CUDA(cudaGetLastError());
            uint32_t more = 0;
            GND_CUDA(cudaMemcpyAsync(&more, qc + (c ^ 1), 4, cudaMemcpyDeviceToHost, st));
            GND_CUDA(cudaStreamSynchronize(st));
            if (more == 0) break;
            std::swap(cur, nxt);
            c ^= 1;
        }
        GND_CUDA(cudaMemcpyAsync(&numBlas, nodeCount, 4, cudaMemcpyDeviceToHost, st));
        GND_CUDA(cudaStreamSynchronize(st));
        if (numBlas > capacity) throw Error(GND_ERR_DEVICE_CHECK, "mesh tree build: node capacity exceeded");
    } else if (M > 0) {
        // meshes without triangles: empty roots
        numBlas = (uint32_t)M;
        blas = PoolBuf((size_t)M * sizeof(Node4), st);
        PoolBuf roots(16, st), qa(16, st), qcount(16, st);
        GND_CUDA(cudaMemsetAsync(qcount.ptr, 0, 16, st));
        kRoots<<<blocksFor((uint64_t)M), kBuildBlock, 0, st>>>(base.as<uint32_t>(), M, roots.as<Slot>(), blas.as<Node4>(),
                                                                qa.as<QEntry>(), qcount.as<uint32_t>());
        GND_CUDA(cudaGetLastError());
    }
    // final node array: top-level nodes, then the mesh trees
    out.numNodes = T + numBlas;
    out.nodes = PoolBuf(std::max<size_t>((size_t)out.numNodes * sizeof(Node4), 16), st);
    if (T) GND_CUDA(cudaMemcpyAsync(out.nodes.ptr, in.tlasNodes, (size_t)T * sizeof(Node4), cudaMemcpyHostToDevice, st));
    if (numBlas)
        GND_CUDA(cudaMemcpyAsync(out.nodes.as<Node4>() + T, blas.ptr, (size_t)numBlas * sizeof(Node4), cudaMemcpyDeviceToDevice, st));
    // 5. leaf order and instance roots
    out.tris = PoolBuf(std::max<size_t>((size_t)N * sizeof(Tri), 16), st);
    out.attrs = PoolBuf(std::max<size_t>((size_t)N * sizeof(TriAttr), 16), st);
    if (N > 0) {
        kGather<<<blocksFor(N), kBuildBlock, 0, st>>>(valsB.as<uint32_t>(), N, in.tris, in.attrs, out.tris.as<Tri>(),
                                                       out.attrs.as<TriAttr>(), in.origToLeaf);
        GND_CUDA(cudaGetLastError());
    }
    if (in.numInstances > 0) {
        kPatch<<<blocksFor((uint64_t)in.numInstances), kBuildBlock, 0, st>>>(in.instT, in.instS, in.numInstances,
                                                                             base.as<uint32_t>(), M, T);
        GND_CUDA(cudaGetLastError());
    }
    GND_CUDA(cudaEventRecord(e1, st));
    uint32_t fl = 0;
    GND_CUDA(cudaMemcpyAsync(&fl, flags.ptr, 4, cudaMemcpyDeviceToHost, st));
    GND_CUDA(cudaStreamSynchronize(st));
    if (fl & kFlagOverflow) throw Error(GND_ERR_DEVICE_CHECK, "mesh tree build: node capacity exceeded");
    out.nonFinite = (fl & kFlagNonFinite) != 0;
    GND_CUDA(cudaEventElapsedTime(&out.ms, e0, e1));
    return out;
}

}  // namespace gnd
