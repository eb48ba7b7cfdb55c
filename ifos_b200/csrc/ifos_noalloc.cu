// ifos_dot_f64_noalloc: the FP64 dot product of ifos_dot_f64 for callers that
// cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code whose GPU memory
// is owned and fully budgeted by another framework (a caching allocator that
// has already reserved the device), a latency-bound loop where cudaMalloc or
// cudaFree would synchronise the whole device, or a pre-allocated inversion
// driver that must not fragment device memory between iterations.  They can
// still reduce data they already hold on the device.  This entry point needs
// no context and touches no allocator: its scratch (one partial sum per block
// plus the result) lives in the file-scope array below, which every GPU that
// loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>

#include "ifos_gpu.h"

// reports through ifos_last_error(NULL) (defined with the context code)
void ifos_internal_set_error(const std::string &msg);

// One partial sum per block in [0, IFOS_NOALLOC_MAX_BLOCKS) and the result at
// IFOS_NOALLOC_MAX_BLOCKS (32 KiB + 8 B on every device that loads the
// library).  Every slot a call reads is written earlier in the same call, so
// nothing has to start at zero.
static __device__ __align__(256) double g_scratch[IFOS_NOALLOC_MAX_BLOCKS + 1];

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = IFOS_NOALLOC_MAX_BLOCKS;
constexpr long long kPerThread = 32;  // elements one thread sums before the block reduction
constexpr int kMaxDevices = 64;

// Device address of g_scratch per device, looked up once with that device
// current (host code must not use the symbol itself as a device pointer).
// Threads making their first call at the same time serialise on the mutex;
// later calls read the published address without locking.
std::atomic<double *> g_scratch_dev[kMaxDevices];
std::mutex g_scratch_mu;

// Restores the calling thread's current device on every return path.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    DeviceGuard() { ok = cudaGetDevice(&prev) == cudaSuccess; }
    ~DeviceGuard() {
        if (ok) cudaSetDevice(prev);
    }
};

__global__ void k_partial(const float *a, const float *b, long long n, double *scratch) {
    double acc = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const double x = a[k];
        acc += x * (b ? (double)b[k] : x);
    }
    __shared__ double red[kThreads / 32];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) scratch[blockIdx.x] = v;
    }
}

// fixed-order sum of the nb partials into scratch[kMaxBlocks]
__global__ void k_final(double *scratch, int nb) {
    __shared__ double red[kThreads / 32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += scratch[k];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) scratch[kMaxBlocks] = v;
    }
}

int fail(int code, const std::string &msg) {
    ifos_internal_set_error(msg);
    return code;
}

}  // namespace

extern "C" int ifos_dot_f64_noalloc(int device, const float *a, const float *b, size_t n, void *stream,
                                    double *out) {
    if (!a || !out) return fail(IFOS_ERR_ARG, "ifos_dot_f64_noalloc: null input or output");
    if (device < 0 || device >= kMaxDevices) return fail(IFOS_ERR_ARG, "ifos_dot_f64_noalloc: bad device index");
    // compared unsigned: a count that wrapped (a negative value through an
    // unsigned parameter) is rejected too, before any launch
    const size_t max_n = (size_t)kMaxBlocks * kThreads * kPerThread;
    if (n > max_n)
        return fail(IFOS_ERR_ARG, "ifos_dot_f64_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                                      std::to_string(max_n) + " elements (" + std::to_string(kMaxBlocks) +
                                      " partial sums of the static scratch)");
    DeviceGuard guard;
    if (!guard.ok) return fail(IFOS_ERR_CUDA, "ifos_dot_f64_noalloc: cudaGetDevice failed");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(IFOS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    double *scratch = g_scratch_dev[device].load(std::memory_order_acquire);
    if (!scratch) {
        // first call on this device: resolve the scratch address (before any capture)
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        scratch = g_scratch_dev[device].load(std::memory_order_relaxed);
        if (!scratch) {
            e = cudaGetSymbolAddress((void **)&scratch, g_scratch);
            if (e != cudaSuccess || !scratch)
                return fail(IFOS_ERR_CUDA,
                            std::string("cudaGetSymbolAddress of the scratch: ") + cudaGetErrorString(e));
            g_scratch_dev[device].store(scratch, std::memory_order_release);
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t per_block = (size_t)kThreads * kPerThread;
    int nb = (int)((n + per_block - 1) / per_block);
    if (nb < 1) nb = 1;
    k_partial<<<nb, kThreads, 0, st>>>(a, b, (long long)n, scratch);
    k_final<<<1, kThreads, 0, st>>>(scratch, nb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch + kMaxBlocks, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(IFOS_ERR_CUDA, std::string("ifos_dot_f64_noalloc: ") + cudaGetErrorString(e));
    return IFOS_OK;
}
