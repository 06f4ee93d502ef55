// Allocation-free reduction for ow3d_residual_device_noalloc (ow3d.cu).
//
// Who needs it: a host that checks the Laplace residual inside its own time
// loop while it owns the device memory budget -- a coupled solver with its own
// pool, or one that must not let a library call cudaMalloc/cudaFree, whose
// implicit device-wide synchronisation would stall its other streams. The
// other ABI calls may allocate (host-pointer calls create staging buffers on
// first use); this path touches no allocator at any call.
//
// Scratch lives in file-scope device arrays of fixed size:
//   g_na_partial  one partial sum per block (kNoAllocBlocks doubles),
//   g_na_counter  blocks finished; must be zero when a launch starts -- it is
//                 zero at module load and the last block of every launch
//                 resets it,
//   g_na_result   the reduced value read back by the host.
// Their addresses are looked up with cudaGetSymbolAddress once per device, on
// the first call made on that device: that first call should come before any
// stream capture begins. Every call reads its result back to the host and
// synchronises the handle's stream before it returns. Two calls that overlap
// in time on one device (different streams or host threads) share this
// scratch and race; callers serialise them.
#include "ow3d_internal.h"

#include <mutex>
#include <string>

namespace ow3d {

namespace {

constexpr int kNoAllocBlocks = 1024;     // partial sums: 8 KB
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_na_partial[kNoAllocBlocks];
static __device__ __align__(256) unsigned int g_na_counter;
static __device__ __align__(256) double g_na_result;

struct Scratch {
    double* partial = nullptr;
    unsigned int* counter = nullptr;
    double* result = nullptr;
};
Scratch g_scratch[kNoAllocMaxDevices];
bool g_ready[kNoAllocMaxDevices] = {};
std::mutex g_mu;

__device__ __forceinline__ double warp_sum_na(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum of squares of y[0..n), one deterministic pass: block partials in a
// fixed order, the last block to finish adds them in index order
__global__ void __launch_bounds__(kNoAllocThreads) k_na_sumsq(const double* __restrict__ y, int n, double* partial,
                                                              unsigned int* counter, double* result) {
    double acc = 0;
    for (int t = blockIdx.x * kNoAllocThreads + threadIdx.x; t < n; t += gridDim.x * kNoAllocThreads) {
        const double v = y[t];
        acc += v * v;
    }
    __shared__ double red[kNoAllocThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    acc = warp_sum_na(acc);
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int q = 0; q < kNoAllocThreads / 32; ++q) s += red[q];
        partial[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (wid == 0) {
        double s = 0;
        for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(partial + b);
        s = warp_sum_na(s);
        if (lane == 0) {
            *result = s;
            *counter = 0u;      // ready for the next launch
        }
    }
}

int scratch_for_device(int dev, Scratch& out, std::string& err) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) { err = "device ordinal out of range for the no-alloc scratch"; return OW3D_ERR_UNSUPPORTED; }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ready[dev]) {
        Scratch s;
        cudaError_t e = cudaGetSymbolAddress((void**)&s.partial, g_na_partial);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.counter, g_na_counter);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.result, g_na_result);
        if (e != cudaSuccess) { err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return OW3D_ERR_CUDA; }
        g_scratch[dev] = s;
        g_ready[dev] = true;
    }
    out = g_scratch[dev];
    return OW3D_OK;
}

}  // namespace

int noalloc_norm2(int dev, const double* d_y, int64_t n, double* host_norm2, cudaStream_t st, std::string& err) {
    if (n < 0 || n > (int64_t)0x7fffffff) {
        err = "no-alloc reduction: vector longer than 2^31-1 elements";
        return OW3D_ERR_UNSUPPORTED;
    }
    Scratch s;
    if (int r = scratch_for_device(dev, s, err)) return r;
    int blocks = (int)((n + kNoAllocThreads - 1) / kNoAllocThreads);
    if (blocks > kNoAllocBlocks) blocks = kNoAllocBlocks;
    if (blocks < 1) blocks = 1;
    note_launch(), k_na_sumsq<<<blocks, kNoAllocThreads, 0, st>>>(d_y, (int)n, s.partial, s.counter, s.result);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { err = std::string("k_na_sumsq: ") + cudaGetErrorString(e); return OW3D_ERR_CUDA; }
    double sumsq = 0;
    e = cudaMemcpyAsync(&sumsq, s.result, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { err = std::string("no-alloc reduction: ") + cudaGetErrorString(e); return OW3D_ERR_CUDA; }
    *host_norm2 = sqrt(sumsq);
    return OW3D_OK;
}

}  // namespace ow3d
