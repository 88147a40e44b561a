// Read-bandwidth probe (gnd_gpu_read_bandwidth): streams a device buffer of a chosen size
// with 16-byte loads that are cached in L2 only, so a buffer smaller than L2 measures L2
// bandwidth and a buffer far larger than L2 measures HBM bandwidth. These are the
// denominators of the traversal roofline.
#include "runtime.h"

namespace gnd {

__global__ void __launch_bounds__(256) kReadProbe(const uint4* __restrict__ p, size_t n16, int reps, uint32_t* sink) {
    uint32_t acc = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r) {
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += stride) {
            const uint4 v = __ldcg(p + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);   // keeps the loads; the buffer is zero
}

}  // namespace gnd

using namespace gnd;

extern "C" {

gnd_status gnd_gpu_read_bandwidth(gnd_gpu_ctx* ctxh, uint64_t bytes, int32_t reps, double* gbps) {
    return guarded([&]() {
        Context* c = ctxOf(ctxh);
        if (!gbps || bytes < 16 || reps <= 0) throw Error(GND_ERR_INVALID, "bad probe arguments");
        c->bind();
        std::lock_guard<FairMutex> lk(c->mu);
        const size_t n16 = (size_t)(bytes / 16);
        DevBuf buf(n16 * 16), sink(sizeof(uint32_t));
        cudaStream_t st = c->stream;
        GND_CUDA(cudaMemsetAsync(buf.ptr, 0, n16 * 16, st));
        GND_CUDA(cudaMemsetAsync(sink.ptr, 0, sizeof(uint32_t), st));
        const int grid = c->numSMs * 8;
        kReadProbe<<<grid, 256, 0, st>>>(buf.as<uint4>(), n16, 1, sink.as<uint32_t>());   // warm-up (fills L2)
        cudaEvent_t e0, e1;
        GND_CUDA(cudaEventCreate(&e0));
        GND_CUDA(cudaEventCreate(&e1));
        GND_CUDA(cudaEventRecord(e0, st));
        kReadProbe<<<grid, 256, 0, st>>>(buf.as<uint4>(), n16, reps, sink.as<uint32_t>());
        GND_CUDA(cudaEventRecord(e1, st));
        GND_CUDA(cudaGetLastError());
        GND_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GND_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *gbps = (double)n16 * 16.0 * reps / (ms * 1e-3) / 1e9;
    });
}

}  // extern "C"
