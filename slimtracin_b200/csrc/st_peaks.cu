// st_peaks.cu — measurement helper of the benchmark (libst_peaks.so), not part of the tracing path.
//
// st_peak_l2_read_gbs: the read bandwidth of the L2 cache, measured on the device.  A buffer that
// fits in L2 (tens of MB against 126 MB) is written once, then read `reps` times by a persistent
// grid of 4 blocks per SM with 128-bit loads that bypass L1 (ld.global.cg), so every load is served
// by L2; the whole sequence is one launch timed with CUDA events.  The figure is the denominator of
// the trace kernel's L2 roofline fraction.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

__global__ void __launch_bounds__(512) l2_read_kernel(const float4 *__restrict__ buf, size_t n4, int reps,
                                                     float *__restrict__ sink) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    float acc = 0.0f;
    for (int r = 0; r < reps; r++) {
        // each pass starts at a rotated offset so that no SM keeps re-reading the same lines
        const size_t start = ((size_t)blockIdx.x * blockDim.x + threadIdx.x + (size_t)r * 9973u * blockDim.x) % stride;
        for (size_t i = start; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    if (acc == 1.2345e-30f) sink[blockIdx.x] = acc;   // keeps the loads; the buffer is all ones
}

__global__ void fill_kernel(float4 *buf, size_t n4) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x)
        buf[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
}

}  // namespace

extern "C" {

// bytes: buffer size (rounded down to 16-byte units); reps: full reads of it in the timed launch.
// Returns 0 and the read rate in GB/s (1e9 bytes per second), or the CUDA error code.
__attribute__((visibility("default"))) int st_peak_l2_read_gbs(int device, uint64_t bytes, int reps, double *gbs) {
    if (!gbs || bytes < 16 || reps < 1) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return (int)e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t n4 = bytes / 16;
    float4 *buf = nullptr;
    float *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int blocks = 4 * (sms > 0 ? sms : 148);
    if ((e = cudaMalloc(&buf, n4 * 16)) != cudaSuccess) return (int)e;
    if ((e = cudaMalloc(&sink, sizeof(float) * blocks)) != cudaSuccess) { cudaFree(buf); return (int)e; }
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fill_kernel<<<blocks, 512>>>(buf, n4);
    l2_read_kernel<<<blocks, 512>>>(buf, n4, 2, sink);          // warm-up: the buffer lands in L2
    cudaEventRecord(e0);
    l2_read_kernel<<<blocks, 512>>>(buf, n4, reps, sink);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) *gbs = (double)n4 * 16.0 * reps / (ms * 1e-3) / 1e9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    cudaFree(buf);
    return (int)e;
}

}  // extern "C"
