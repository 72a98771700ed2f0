// Reduction entry point that allocates nothing (C ABI: pb_reduce_noalloc_f64).
//
// pb_reduce_f64 / pb_reduce_async_f64 obtain their scratch (per-block partial results and a
// completion ticket) with cudaMalloc on their first call on a device. Some callers cannot allow
// that: code running while a CUDA stream is being captured into a graph (a cudaMalloc there breaks
// the capture), applications whose device memory is entirely owned by another allocator or a
// fixed budget, and runtimes that must not grow device memory after start-up. This variant keeps
// its scratch in a file-scope static __device__ array instead, which every GPU that loads the
// library holds until the process exits.
//
// Scheme: block b folds the fixed chunk [b*kChunk, (b+1)*kChunk) of the region (flattened x
// fastest) into partial b; the last block to finish (atomic ticket) folds the partials in block
// order and writes the result, so results do not depend on the GPU's size. The scratch holds
// kMaxChunks partials, which bounds the region volume at kMaxChunks * kChunk elements.
#include <cfloat>
#include <cstring>

#include "pb_internal.cuh"

namespace pb {
namespace noalloc {

constexpr int kThreads = 256;
constexpr long long kChunk = 2048;                 // elements per block
constexpr int kMaxChunks = 4096;                   // partial slots held by the static scratch
constexpr long long kMaxElems = kChunk * kMaxChunks;
constexpr size_t kScratchBytes = kMaxChunks * sizeof(double) + 256;   // partials, then the ticket

// The scratch: shared by every call on a device; calls that overlap on the GPU race on it.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__device__ __forceinline__ double init_of(int op) { return op == 0 ? DBL_MIN : op == 1 ? DBL_MAX : 0.0; }
__device__ __forceinline__ double fold(int op, double a, double v)
{
    switch (op) {
        case 0: return (a < v) ? v : a;
        case 1: return (v < a) ? v : a;
        case 2: return upd_abs(a, v);
        case 3: return dadd(a, v);
        case 4: return dadd(a, v > 0 ? v : -v);
        default: return dadd(a, dmul(v, v));
    }
}
__device__ __forceinline__ double comb(int op, double a, double b)
{
    switch (op) {
        case 0: case 2: return (a < b) ? b : a;
        case 1: return (b < a) ? b : a;
        default: return dadd(a, b);
    }
}
__device__ double block_comb(int op, double v)
{
    __shared__ double sh[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = comb(op, v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[lane] : init_of(op);
    if (wid == 0)
        for (int o = 16; o > 0; o >>= 1) v = comb(op, v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(kThreads) k_reduce_chunks(int op, const double* __restrict__ data, Box3 b, int rlo0,
                                                             int rlo1, int rlo2, int rn0, int rn1, long long total,
                                                             unsigned char* scratch, double* result)
{
    double* partials = reinterpret_cast<double*>(scratch);
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kMaxChunks * sizeof(double));
    const long long Sx = bsize(b, 0), Sxy = bsize(b, 0) * bsize(b, 1);
    const long long begin = (long long)blockIdx.x * kChunk;
    const long long end = begin + kChunk < total ? begin + kChunk : total;
    double v = init_of(op);
    for (long long i = begin + threadIdx.x; i < end; i += blockDim.x) {
        int x = rlo0 + (int)(i % rn0);
        long long q = i / rn0;
        int y = rlo1 + (int)(q % rn1);
        int z = rlo2 + (int)(q / rn1);
        v = fold(op, v, data[(x - b.lo[0]) + Sx * (y - b.lo[1]) + Sxy * (z - b.lo[2])]);
    }
    v = block_comb(op, v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double w = init_of(op);
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
        double p = ((volatile double*)partials)[k];
        w = (k == (int)threadIdx.x) ? p : comb(op, w, p);
    }
    w = block_comb(op, w);
    if (threadIdx.x == 0) {
        *result = w;
        *ticket = 0;
    }
}

// Device address of g_scratch per device ordinal, resolved once with that device current. The cache
// lives as long as the process's CUDA context on that device: after cudaDeviceReset the module may be
// loaded again at another address, so a caller that resets a device must not call this entry point
// on it again in the same process. Two host threads that race on a device's first call both store
// the same address, which is harmless.
static unsigned char* g_addr[64] = {nullptr};

static int scratch_address(unsigned char** out)
{
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return PB_ERR_UNSUPPORTED;
    if (!g_addr[dev]) {
        void* p = nullptr;
        PB_CUDA(cudaGetSymbolAddress(&p, g_scratch));
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return PB_OK;
}

} // namespace noalloc
} // namespace pb

using namespace pb;

extern "C" int pb_reduce_noalloc_f64(int op, const double* data, pb_box box, pb_box region, double* result_dev,
                                     void* stream)
{
    if (!data || !result_dev || op < 0 || op > 5) return PB_ERR_ARG;
    Box3 b = to_box(box), r = to_box(region);
    if (bempty(b)) return PB_ERR_BOX;
    r = bempty(r) ? b : intersect(r, b);
    long long total = bempty(r) ? 0 : bvol(r);
    if (total > noalloc::kMaxElems) return PB_ERR_BUDGET;   // more partials than the static scratch holds
    unsigned char* scratch = nullptr;
    int e = noalloc::scratch_address(&scratch);
    if (e != PB_OK) return e;
    cudaStream_t st = (cudaStream_t)stream;
    // the ticket must start at zero: clear it on the stream (no allocation involved)
    PB_CUDA(cudaMemsetAsync(scratch + noalloc::kMaxChunks * sizeof(double), 0, sizeof(unsigned int), st));
    int blocks = (int)((total + noalloc::kChunk - 1) / noalloc::kChunk);
    if (blocks < 1) blocks = 1;
    int rlo[3] = {0, 0, 0}, rn[3] = {1, 1, 1};
    if (total > 0)
        for (int d = 0; d < 3; d++) { rlo[d] = r.lo[d]; rn[d] = (int)bsize(r, d); }
    noalloc::k_reduce_chunks<<<blocks, noalloc::kThreads, 0, st>>>(op, data, b, rlo[0], rlo[1], rlo[2], rn[0], rn[1],
                                                                   total, scratch, result_dev);
    PB_LAUNCH_CHECK();
    return PB_OK;
}
