// pt_probe.cu — read-bandwidth probe (sm_100a).
//
// The traversal kernels mostly read (tree nodes, triangle records, rays) from a working set that
// lives in L2 for the 1M-triangle scene and in HBM for larger ones.  This probe measures the
// read bandwidth of this GPU for a buffer of a given size with the same 16-byte vector loads:
// a buffer well under the 126 MB L2 gives the L2 read bandwidth, one of several GB the HBM read
// bandwidth.  The roofline of the traversal is quoted against both.
#include <algorithm>
#include "pt_api_common.h"
#include "pt_device.h"

using namespace ptb;

namespace {

// Each thread sums every gridDim*blockDim-th float4 of the buffer, `reps` times over; the sum is
// stored only when it equals a value it cannot take, so the loads are not removed.
__global__ void __launch_bounds__(512) read_probe_kernel(const float4 *__restrict__ data, size_t n4, int reps, float *sink) {
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    float acc = 0.0f;
    for (int r = 0; r < reps; r++) {
        size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
        for (; i + 3 * stride < n4; i += 4 * stride) {
            float4 a = __ldcg(data + i), b = __ldcg(data + i + stride), c = __ldcg(data + i + 2 * stride), d = __ldcg(data + i + 3 * stride);
            acc += (a.x + a.y + a.z + a.w) + (b.x + b.y + b.z + b.w) + (c.x + c.y + c.z + c.w) + (d.x + d.y + d.z + d.w);
        }
        for (; i < n4; i += stride) {
            float4 a = __ldcg(data + i);
            acc += a.x + a.y + a.z + a.w;
        }
    }
    if (acc == -1.0f) sink[0] = acc;
}

} // namespace

extern "C" {

// Read bandwidth (GB/s, 1e9 bytes per second) over a buffer of `bytes` (rounded down to 16 bytes,
// zero-filled), read `reps` times inside one launch after one untimed warm-up launch.
pt_status pt_probe_read_bandwidth(size_t bytes, int reps, float *gbs) {
    return guard([&]() {
        if (!gbs || bytes < 16 || reps < 1) throw Error(PT_INVALID_ARGUMENT, "invalid probe arguments");
        require_device();
        const size_t n4 = bytes / 16;
        DeviceBuffer buf(n4 * 16), sink(sizeof(float));
        PT_CUDA(cudaMemset(buf.get(), 0, n4 * 16));
        const int sms = device_sm_count();
        const unsigned grid = unsigned(sms) * 4u;
        read_probe_kernel<<<grid, 512>>>(buf.get<float4>(), n4, 1, sink.get<float>());
        PT_CUDA(cudaGetLastError());
        Event start, stop;
        PT_CUDA(cudaEventRecord(start.get()));
        read_probe_kernel<<<grid, 512>>>(buf.get<float4>(), n4, reps, sink.get<float>());
        PT_CUDA(cudaEventRecord(stop.get()));
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaEventSynchronize(stop.get()));
        float ms = 0;
        PT_CUDA(cudaEventElapsedTime(&ms, start.get(), stop.get()));
        *gbs = float(double(n4) * 16.0 * reps / (double(ms) * 1e-3) / 1e9);
    });
}

} // extern "C"
