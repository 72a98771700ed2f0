// Shared internals of the sm_100a structured-grid library: boxes, status handling, the
// device error flag, exact-rounding arithmetic helpers, and TMA / mbarrier wrappers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/proto_b200.h"

namespace pb {

// ---------------------------------------------------------------------------------------------
// Host-side status plumbing
// ---------------------------------------------------------------------------------------------
void set_cuda_error(cudaError_t e);
#define PB_CUDA(call)                                   \
    do {                                                \
        cudaError_t e__ = (call);                       \
        if (e__ != cudaSuccess) {                       \
            ::pb::set_cuda_error(e__);                  \
            return PB_ERR_CUDA;                         \
        }                                               \
    } while (0)
#define PB_LAUNCH_CHECK() PB_CUDA(cudaGetLastError())

// ---------------------------------------------------------------------------------------------
// Boxes (Proto::Box semantics: inclusive corners, x-fastest linear index)
// ---------------------------------------------------------------------------------------------
struct Box3 {
    int lo[3], hi[3];
};
inline Box3 to_box(const pb_box& b)
{
    Box3 r;
    for (int d = 0; d < 3; d++) { r.lo[d] = b.lo[d]; r.hi[d] = b.hi[d]; }
    return r;
}
__host__ __device__ inline long long bsize(const Box3& b, int d) { return (long long)b.hi[d] - b.lo[d] + 1; }
__host__ __device__ inline bool bempty(const Box3& b)
{
    return b.hi[0] < b.lo[0] || b.hi[1] < b.lo[1] || b.hi[2] < b.lo[2];
}
__host__ __device__ inline long long bvol(const Box3& b)
{
    return bempty(b) ? 0 : bsize(b, 0) * bsize(b, 1) * bsize(b, 2);
}
inline Box3 intersect(const Box3& a, const Box3& b)
{
    Box3 r;
    for (int d = 0; d < 3; d++) {
        r.lo[d] = a.lo[d] > b.lo[d] ? a.lo[d] : b.lo[d];
        r.hi[d] = a.hi[d] < b.hi[d] ? a.hi[d] : b.hi[d];
    }
    return r;
}
inline bool contains_box(const Box3& outer, const Box3& inner)
{
    if (bempty(inner)) return true;
    for (int d = 0; d < 3; d++)
        if (inner.lo[d] < outer.lo[d] || inner.hi[d] > outer.hi[d]) return false;
    return true;
}
// Point division rounds toward -infinity (Proto_PointImplem.H:212-239)
__host__ __device__ inline int floor_div(int a, int r) { int q = a / r; return (a % r != 0 && ((a < 0) != (r < 0))) ? q - 1 : q; }
__host__ __device__ inline int ceil_div(int a, int r) { int q = a / r; return (a % r != 0 && ((a < 0) == (r < 0))) ? q + 1 : q; }
// Box::taperCoarsen (Proto_BoxImplem.H:555-564): high = floor(hi/r), low = ceil(lo/r)
inline Box3 taper_coarsen(const Box3& b, const int* r)
{
    Box3 o;
    for (int d = 0; d < 3; d++) {
        o.hi[d] = floor_div(b.hi[d], r[d]);
        o.lo[d] = ceil_div(b.lo[d], r[d]);
    }
    return o;
}

// ---------------------------------------------------------------------------------------------
// Device error flag: kernels set it instead of trapping; pb_device_check reads and clears it.
// ---------------------------------------------------------------------------------------------
// The flag is per translation unit (no relocatable device code); every .cu file that launches a
// kernel able to flag an error defines a reader with PB_DEFINE_ERROR_READER.
enum DeviceError : int { DEV_OK = 0, DEV_WAIT_TIMEOUT = 1, DEV_BAD_INDEX = 2 };
static __device__ int g_dev_error = 0;
__device__ inline void flag_error(int code) { atomicCAS(&g_dev_error, 0, code); }
#define PB_DEFINE_ERROR_READER(name)                                                   \
    int name()                                                                         \
    {                                                                                  \
        int flag = 0, zero = 0;                                                        \
        if (cudaMemcpyFromSymbol(&flag, g_dev_error, sizeof(int)) != cudaSuccess) return -1; \
        if (flag) cudaMemcpyToSymbol(g_dev_error, &zero, sizeof(int));                 \
        return flag;                                                                   \
    }
int read_error_stencil();
int read_error_mg();
int read_error_serve();
int read_error_fas();

// ---------------------------------------------------------------------------------------------
// Exact arithmetic: one IEEE rounding per operation, never contracted into FMA (FP32 sums: dmadd)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float dmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float dsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ddiv(float a, float b) { return __fdiv_rn(a, b); }
// acc + a*b, the step of every stencil, restriction and smoother sum: FP64 rounds the product and
// the sum separately (the reference's arithmetic, bit for bit); FP32 (mixed-precision cycles and the
// FP32 API, not held to the reference's rounding) takes one fused multiply-add, half the instructions
// of the issue-bound FP32 sweeps. Every FP32 level kernel, single-solve and served, uses it, so their
// results stay bitwise equal to one another.
__device__ __forceinline__ double dmadd(double acc, double a, double b) { return __dadd_rn(acc, __dmul_rn(a, b)); }
__device__ __forceinline__ float dmadd(float acc, float a, float b) { return __fmaf_rn(a, b, acc); }
// the quotient of a Jacobi update: FP64 keeps the correctly rounded division (the reference's
// arithmetic, bit for bit); FP32 (mixed-precision cycles, whose error the FP64 residual and
// correction remove) takes the reciprocal-multiply form (within 2 ulp), two instructions instead
// of the correctly rounded division's sequence
__device__ __forceinline__ double squot(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float squot(float a, float b) { return __fdividef(a, b); }

// Reduction<T,Abs>::update (Proto_ReductionImplem.H:87): NaN inputs leave the value unchanged.
__device__ __forceinline__ double upd_abs(double v1, double v2)
{
    double a = v2 > 0 ? v2 : -v2;
    return (v1 < a) ? a : v1;
}
// atomic max of a non-negative double through its bit pattern (monotone for x >= 0)
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v)
{
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// ---------------------------------------------------------------------------------------------
// mbarrier + TMA (sm_90+ PTX; every wait is bounded)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// per-thread asynchronous global -> shared copies (8 or 16 bytes), grouped and waited on per group
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: returns false (and flags DEV_WAIT_TIMEOUT) if the phase has not completed after
// `tries` polls. Every pipelined kernel waits through mbar_wait (kMaxWaitTries polls, about a
// second); pb_debug_wait_expiry runs the same code with a small limit so a test can make it expire.
constexpr uint32_t kMaxWaitTries = 1u << 24;
__device__ __forceinline__ bool mbar_wait_limited(uint64_t* bar, uint32_t parity, uint32_t tries)
{
    for (uint32_t i = 0; i < tries; i++)
        if (mbar_try_wait(bar, parity)) return true;
    flag_error(DEV_WAIT_TIMEOUT);
    return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    return mbar_wait_limited(bar, parity, kMaxWaitTries);
}
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Host: encode a 3-D tiled tensor map over a field on a box (dims Sx,Sy,Sz elements of esize).
// Returns PB_OK, PB_ERR_ALIGN when the TMA rules (16-byte base, 16-byte strides) are not met.
int encode_tmap_3d(CUtensorMap* map, const void* base, int esize, long long Sx, long long Sy, long long Sz,
                   int boxX, int boxY, int boxZ);
bool tma_available();

} // namespace pb
