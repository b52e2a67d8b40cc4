// Body segmentation with no device allocation.
//
// Some callers cannot allocate device memory at the moment they need this: code that runs while a CUDA
// stream is being captured into a graph (cudaMalloc is not a capturable operation and fails the capture), a
// host application that hands the GPU's memory to its own pool and forbids other allocations (a renderer or a
// DCC plug-in sharing the device), or a caller on a latency-critical path that cannot afford the implicit
// device synchronisation of cudaMalloc / cudaFree.  For them this entry point runs the library's body
// segmentation on caller-owned input and output buffers, with all working memory in one file-scope device
// array that the library image carries.
//
// That array is a fixed 16 MB per GPU, held by every GPU that loads the library until the process exits, and
// limits a call to kNoAllocMaxParticles particles.  Every call shares it and leaves its contents behind; the
// entry point clears the parts that must start at zero on each call.  Two calls that overlap on the GPU (on
// different streams, or from different host threads) use the same array and race; serialise them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/mpm_gpu.h"
#include "mpm_kernels.h"
#include "mpm_types.h"

namespace {

constexpr int kNoAllocMaxParticles = 1 << 18;  // 262,144
constexpr int kNoAllocHashBits = 19;           // 2^19 hash buckets = 2 per particle at the maximum
constexpr size_t kBuckets = size_t(1) << kNoAllocHashBits;
constexpr size_t kScanTmp = 4096;               // ints; covers the recursive scan of 2^19 elements
// layout: [bucket count | bucket start] [8 int arrays of kNoAllocMaxParticles] [scalars(16) | scan tmp]
//         [positions in bucket order: float4 x max] [zero velocities: 3 floats x max]
constexpr size_t kIntsBuckets = 2 * kBuckets;
constexpr size_t kIntsParticles = 8 * size_t(kNoAllocMaxParticles);
constexpr size_t kIntsTail = 16 + kScanTmp;
constexpr size_t kIntBytes = (kIntsBuckets + kIntsParticles + kIntsTail) * sizeof(int);
constexpr size_t kXsOffset = (kIntBytes + 255) / 256 * 256;
constexpr size_t kVOffset = kXsOffset + sizeof(float4) * kNoAllocMaxParticles;
constexpr size_t kScratchBytes = kVOffset + 3 * sizeof(float) * kNoAllocMaxParticles;

__device__ __align__(256) unsigned char g_segScratch[kScratchBytes];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
    CUcontext ctx;   // the context the address belongs to
    void* addr;
};
ScratchAddr g_scratch[kMaxDevices] = {};
std::mutex g_scratchMutex;

// The current context (the driver's cuCtxGetCurrent, reached through the runtime so that the library does not
// link the driver library); null if it cannot be queried.
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return reinterpret_cast<Fn>(p);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of g_segScratch on the current device.  Set up once per device, with that device current
// (cudaGetSymbolAddress loads the library's module on the device the first time, which is what places the
// array there), and again if the device's context changed since: after cudaDeviceReset the module is loaded
// anew and the array may sit at another address.
cudaError_t scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    ScratchAddr& s = g_scratch[dev];
    const CUcontext ctx = current_context();
    if (!s.addr || !ctx || ctx != s.ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_segScratch);
        if (e != cudaSuccess) return e;
        s.addr = p;
        s.ctx = current_context();  // the primary context exists now, if it did not before
    }
    *out = s.addr;
    return cudaSuccess;
}

__global__ void k_noalloc_iota(int* a, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

}  // namespace

extern "C" {

int mpm_calculate_bodies_noalloc_max(void) { return kNoAllocMaxParticles; }

mpm_status mpm_calculate_bodies_noalloc(const float* x_device, size_t n, float grid_size, int* body_device,
                                        int* counts_device, void* stream) {
    if (n > (size_t)kNoAllocMaxParticles) return MPM_ERR_TOO_MANY_PARTICLES;
    if ((n > 0 && (!x_device || !body_device)) || !counts_device || !(grid_size > 0.f)) return MPM_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return MPM_ERR_CUDA;
    const int N = (int)n;
    if (N == 0) {
        return cudaMemsetAsync(counts_device, 0, 2 * sizeof(int), s) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
    }
    int* ip = static_cast<int*>(base);
    mpm::SegArrays S{};
    S.count = ip;
    S.start = ip + kBuckets;
    int* pa = ip + kIntsBuckets;
    S.sorted = pa + 0 * size_t(kNoAllocMaxParticles);
    S.rank = pa + 1 * size_t(kNoAllocMaxParticles);
    S.parent = pa + 2 * size_t(kNoAllocMaxParticles);
    S.size = pa + 3 * size_t(kNoAllocMaxParticles);
    S.minOrig = pa + 4 * size_t(kNoAllocMaxParticles);
    S.mark = pa + 5 * size_t(kNoAllocMaxParticles);
    S.mrank = pa + 6 * size_t(kNoAllocMaxParticles);
    int* orig = pa + 7 * size_t(kNoAllocMaxParticles);
    // [0] bodies [1] ballistic [2] scan total [3] error bits [4..9] the particles' bounding box
    int* scalars = ip + kIntsBuckets + kIntsParticles;
    int* scanTmp = scalars + 16;
    S.nbodies = scalars;
    S.bbox = reinterpret_cast<unsigned int*>(scalars + 4);
    S.xs = reinterpret_cast<float4*>(static_cast<unsigned char*>(base) + kXsOffset);
    float* zeroV = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + kVOffset);

    int bits = 10;
    while ((1ll << bits) < 2ll * N && bits < kNoAllocHashBits) ++bits;
    if (mpm::scan_tmp_ints(std::max<long long>(1ll << bits, N)) > kScanTmp) return MPM_ERR_INTERNAL;

    // what must start at zero: the velocity stand-in (read by the NaN check) and the error bits; the
    // segmentation clears its own counters, sizes and marks
    if (cudaMemsetAsync(zeroV, 0, 3 * sizeof(float) * (size_t)N, s) != cudaSuccess) return MPM_ERR_CUDA;
    if (cudaMemsetAsync(scalars, 0, 16 * sizeof(int), s) != cudaSuccess) return MPM_ERR_CUDA;
    k_noalloc_iota<<<(N + 255) / 256, 256, 0, s>>>(orig, N);

    mpm::PartArrays P{};
    P.x = const_cast<float*>(x_device);
    P.v = zeroV;
    P.orig = orig;
    P.body = body_device;
    mpm::launch_segment(P, N, grid_size, S, bits, scanTmp, scalars + 3, s);
    if (cudaMemcpyAsync(counts_device, scalars, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess) return MPM_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

}  // extern "C"
