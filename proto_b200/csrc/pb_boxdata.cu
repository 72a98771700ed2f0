// BoxData algebra, copyTo, pointwise (forall) kernels, reductions and constant prolongation.
//
// Reference counterparts (paths within the reference project):
//   BoxData::operatorT / scalar ops ... include/base/implem/Proto_BoxDataImplem.H:860-985, 1086-1110
//   BoxData::copyTo (general) ......... include/base/implem/Proto_BoxDataImplem.H:493-640
//   forall / forallInPlace ............ include/base/implem/Proto_ForallImplem.H:178-389
//   Reduction<T,OP,DEVICE> ............ include/base/Proto_Reduction.H:113-185,
//                                       include/base/implem/Proto_ReductionImplem.H:108-192
//   InterpStencil::Constant ........... include/base/implem/Proto_InterpStencilDefs.H:1-15
// The reference launches one kernel per call with blocks of one x-row each; these kernels are
// grid-stride loops over the flattened box with coalesced x-fastest accesses.
#include <cfloat>
#include <cstring>

#include "pb_internal.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

struct Region {
    int lo[3];
    int n[3];
};

// ---- dst op= src on a region (both fields addressed through their own boxes) -----------------
template <int OP>
__global__ void __launch_bounds__(256) k_binop(double* dst, Box3 db, const double* __restrict__ src, Box3 sb, Region r,
                                               int shx, int shy, int shz, int ncomp)
{
    const long long total = (long long)r.n[0] * r.n[1] * r.n[2];
    const long long dSx = bsize(db, 0), dSxy = bsize(db, 0) * bsize(db, 1), dvol = bvol(db);
    const long long sSx = bsize(sb, 0), sSxy = bsize(sb, 0) * bsize(sb, 1), svol = bvol(sb);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = r.lo[0] + (int)(i % r.n[0]);
        long long q = i / r.n[0];
        int y = r.lo[1] + (int)(q % r.n[1]);
        int z = r.lo[2] + (int)(q / r.n[1]);
        // (x,y,z) is a source point; its destination is shifted
        long long si = (x - sb.lo[0]) + sSx * (y - sb.lo[1]) + sSxy * (z - sb.lo[2]);
        long long di = (x + shx - db.lo[0]) + dSx * (y + shy - db.lo[1]) + dSxy * (z + shz - db.lo[2]);
        for (int c = 0; c < ncomp; c++) {
            double s = src[si + c * svol];
            double& d = dst[di + c * dvol];
            if (OP == PB_OP_ADD) d = dadd(d, s);
            else if (OP == PB_OP_SUB) d = dsub(d, s);
            else if (OP == PB_OP_MUL) d = dmul(d, s);
            else if (OP == PB_OP_DIV) d = ddiv(d, s);
            else d = s;
        }
    }
}

template <int OP>
__global__ void __launch_bounds__(256) k_scalar(double* dst, Box3 db, Region r, double v, int ncomp)
{
    const long long total = (long long)r.n[0] * r.n[1] * r.n[2];
    const long long dSx = bsize(db, 0), dSxy = bsize(db, 0) * bsize(db, 1), dvol = bvol(db);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = r.lo[0] + (int)(i % r.n[0]);
        long long q = i / r.n[0];
        int y = r.lo[1] + (int)(q % r.n[1]);
        int z = r.lo[2] + (int)(q / r.n[1]);
        long long di = (x - db.lo[0]) + dSx * (y - db.lo[1]) + dSxy * (z - db.lo[2]);
        for (int c = 0; c < ncomp; c++) {
            double& d = dst[di + c * dvol];
            if (OP == PB_OP_ADD) d = dadd(d, v);
            else if (OP == PB_OP_SUB) d = dsub(d, v);
            else if (OP == PB_OP_MUL) d = dmul(d, v);
            else if (OP == PB_OP_DIV) d = ddiv(d, v);
            else d = v;
        }
    }
}

// forall body "out = a*x + b*y" (config: out = a*L(u) + b*u when Lu is materialised)
__global__ void __launch_bounds__(256) k_axpby(double* out, Box3 ob, const double* __restrict__ xs, Box3 xb,
                                               const double* __restrict__ ys, Box3 yb, Region r, double a, double b)
{
    const long long total = (long long)r.n[0] * r.n[1] * r.n[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = r.lo[0] + (int)(i % r.n[0]);
        long long q = i / r.n[0];
        int y = r.lo[1] + (int)(q % r.n[1]);
        int z = r.lo[2] + (int)(q / r.n[1]);
        long long oi = (x - ob.lo[0]) + bsize(ob, 0) * ((y - ob.lo[1]) + bsize(ob, 1) * (long long)(z - ob.lo[2]));
        long long xi = (x - xb.lo[0]) + bsize(xb, 0) * ((y - xb.lo[1]) + bsize(xb, 1) * (long long)(z - xb.lo[2]));
        long long yi = (x - yb.lo[0]) + bsize(yb, 0) * ((y - yb.lo[1]) + bsize(yb, 1) * (long long)(z - yb.lo[2]));
        out[oi] = dadd(dmul(a, xs[xi]), dmul(b, ys[yi]));
    }
}

// ---- reductions ---------------------------------------------------------------------------------
// Pass 1: every block folds its grid-stride share; pass 2 (the last block to finish, found through
// an atomic ticket) folds the per-block partials in block order, so sums are deterministic.
constexpr int kRedBlocks = 1024;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double red_init(int op)
{
    return op == 0 ? DBL_MIN : op == 1 ? DBL_MAX : 0.0;
}
__device__ __forceinline__ double red_upd(int op, double v1, double v2)
{
    switch (op) {
        case 0: return (v1 < v2) ? v2 : v1;                 // std::max
        case 1: return (v2 < v1) ? v2 : v1;                 // std::min
        case 2: return upd_abs(v1, v2);
        case 3: return dadd(v1, v2);
        case 4: return dadd(v1, v2 > 0 ? v2 : -v2);
        default: return dadd(v1, dmul(v2, v2));
    }
}
// combining two partial results (for Abs/SumAbs/SumSquare the partials are already folded)
__device__ __forceinline__ double red_comb(int op, double a, double b)
{
    switch (op) {
        case 0: return (a < b) ? b : a;
        case 1: return (b < a) ? b : a;
        case 2: return (a < b) ? b : a;
        default: return dadd(a, b);
    }
}

__device__ double block_reduce(int op, double v)
{
    __shared__ double sh[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = red_comb(op, v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[lane] : red_init(op == 2 ? 2 : op);
    if (wid == 0)
        for (int o = 16; o > 0; o >>= 1) v = red_comb(op, v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(kRedThreads) k_reduce(int op, const double* __restrict__ data, Box3 b, Region r,
                                                        double* partials, unsigned int* ticket, double* result)
{
    const long long total = (long long)r.n[0] * r.n[1] * r.n[2];
    const long long Sx = bsize(b, 0), Sxy = bsize(b, 0) * bsize(b, 1);
    double v = red_init(op);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = r.lo[0] + (int)(i % r.n[0]);
        long long q = i / r.n[0];
        int y = r.lo[1] + (int)(q % r.n[1]);
        int z = r.lo[2] + (int)(q / r.n[1]);
        v = red_upd(op, v, data[(x - b.lo[0]) + Sx * (y - b.lo[1]) + Sxy * (z - b.lo[2])]);
    }
    v = block_reduce(op, v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double w = red_init(op);
    // fixed order over the partials: thread k folds partials k, k+256, ... then the block tree
    for (int k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        double p = ((volatile double*)partials)[k];
        w = (k == threadIdx.x) ? p : red_comb(op, w, p);
    }
    if (threadIdx.x >= gridDim.x) w = red_init(op);
    w = block_reduce(op, w);
    if (threadIdx.x == 0) {
        *result = w;
        *ticket = 0;
    }
}

// ---- piecewise-constant prolongation ----------------------------------------------------------
__global__ void __launch_bounds__(256) k_interp_const(int ratio, const double* __restrict__ src, Box3 sb, double* dst,
                                                      Box3 db, Region r, int overwrite, double scale)
{
    const long long total = (long long)r.n[0] * r.n[1] * r.n[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = r.lo[0] + (int)(i % r.n[0]);
        long long q = i / r.n[0];
        int y = r.lo[1] + (int)(q % r.n[1]);
        int z = r.lo[2] + (int)(q / r.n[1]);
        int cx = floor_div(x, ratio), cy = floor_div(y, ratio), cz = floor_div(z, ratio);
        double v = src[(cx - sb.lo[0]) + bsize(sb, 0) * ((cy - sb.lo[1]) + bsize(sb, 1) * (long long)(cz - sb.lo[2]))];
        long long di = (x - db.lo[0]) + bsize(db, 0) * ((y - db.lo[1]) + bsize(db, 1) * (long long)(z - db.lo[2]));
        double acc = overwrite ? 0.0 : dst[di];
        dst[di] = dadd(acc, dmul(scale, v));
    }
}

// ---- reduction scratch (per process, per device 0..15) ----------------------------------------
struct RedScratch {
    double* partials = nullptr;
    unsigned int* ticket = nullptr;
    double* result = nullptr;
};
static RedScratch g_red[16];

static int red_scratch(RedScratch** out)
{
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) return PB_ERR_UNSUPPORTED;
    RedScratch& s = g_red[dev];
    if (!s.partials) {
        PB_CUDA(cudaMalloc(&s.partials, kRedBlocks * sizeof(double)));
        PB_CUDA(cudaMalloc(&s.ticket, sizeof(unsigned int)));
        PB_CUDA(cudaMemset(s.ticket, 0, sizeof(unsigned int)));
        PB_CUDA(cudaMalloc(&s.result, sizeof(double)));
    }
    *out = &s;
    return PB_OK;
}

static inline Region region_of(const Box3& b)
{
    Region r;
    for (int d = 0; d < 3; d++) { r.lo[d] = b.lo[d]; r.n[d] = (int)bsize(b, d); }
    return r;
}

} // namespace pb

using namespace pb;

extern "C" {

int pb_boxdata_op_f64(int op, double* dst, pb_box dst_box, const double* src, pb_box src_box, int ncomp, void* stream)
{
    if (!dst || !src || ncomp < 1 || op < 0 || op > PB_OP_ASSIGN) return PB_ERR_ARG;
    Box3 db = to_box(dst_box), sb = to_box(src_box);
    Box3 r = intersect(db, sb);
    if (bempty(r)) return PB_OK;
    Region rg = region_of(r);
    cudaStream_t st = (cudaStream_t)stream;
    int grid = grid_for(bvol(r), 256);
    switch (op) {
        case PB_OP_ADD: k_binop<PB_OP_ADD><<<grid, 256, 0, st>>>(dst, db, src, sb, rg, 0, 0, 0, ncomp); break;
        case PB_OP_SUB: k_binop<PB_OP_SUB><<<grid, 256, 0, st>>>(dst, db, src, sb, rg, 0, 0, 0, ncomp); break;
        case PB_OP_MUL: k_binop<PB_OP_MUL><<<grid, 256, 0, st>>>(dst, db, src, sb, rg, 0, 0, 0, ncomp); break;
        case PB_OP_DIV: k_binop<PB_OP_DIV><<<grid, 256, 0, st>>>(dst, db, src, sb, rg, 0, 0, 0, ncomp); break;
        default: k_binop<PB_OP_ASSIGN><<<grid, 256, 0, st>>>(dst, db, src, sb, rg, 0, 0, 0, ncomp); break;
    }
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_boxdata_scalar_f64(int op, double* dst, pb_box dst_box, pb_box region, double scalar, int ncomp, void* stream)
{
    if (!dst || ncomp < 1 || op < 0 || op > PB_OP_ASSIGN) return PB_ERR_ARG;
    Box3 db = to_box(dst_box), r = to_box(region);
    if (bempty(db)) return PB_ERR_BOX;
    r = bempty(r) ? db : intersect(r, db);
    if (bempty(r)) return PB_OK;
    Region rg = region_of(r);
    cudaStream_t st = (cudaStream_t)stream;
    int grid = grid_for(bvol(r), 256);
    switch (op) {
        case PB_OP_ADD: k_scalar<PB_OP_ADD><<<grid, 256, 0, st>>>(dst, db, rg, scalar, ncomp); break;
        case PB_OP_SUB: k_scalar<PB_OP_SUB><<<grid, 256, 0, st>>>(dst, db, rg, scalar, ncomp); break;
        case PB_OP_MUL: k_scalar<PB_OP_MUL><<<grid, 256, 0, st>>>(dst, db, rg, scalar, ncomp); break;
        case PB_OP_DIV: k_scalar<PB_OP_DIV><<<grid, 256, 0, st>>>(dst, db, rg, scalar, ncomp); break;
        default: k_scalar<PB_OP_ASSIGN><<<grid, 256, 0, st>>>(dst, db, rg, scalar, ncomp); break;
    }
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_boxdata_copy_f64(const double* src, pb_box src_box, double* dst, pb_box dst_box, pb_box src_region,
                        const int shift[3], int ncomp, void* stream)
{
    if (!dst || !src || ncomp < 1) return PB_ERR_ARG;
    Box3 sb = to_box(src_box), db = to_box(dst_box), r = to_box(src_region);
    int sh[3] = {shift ? shift[0] : 0, shift ? shift[1] : 0, shift ? shift[2] : 0};
    r = bempty(r) ? sb : intersect(r, sb);
    Box3 dshift;
    for (int d = 0; d < 3; d++) { dshift.lo[d] = db.lo[d] - sh[d]; dshift.hi[d] = db.hi[d] - sh[d]; }
    r = intersect(r, dshift);
    if (bempty(r)) return PB_OK;
    Region rg = region_of(r);
    k_binop<PB_OP_ASSIGN><<<grid_for(bvol(r), 256), 256, 0, (cudaStream_t)stream>>>(dst, db, src, sb, rg, sh[0], sh[1],
                                                                                   sh[2], ncomp);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_forall_axpby_f64(double* out, pb_box out_box, const double* x, pb_box x_box, const double* y, pb_box y_box,
                        double a, double b, void* stream)
{
    if (!out || !x || !y) return PB_ERR_ARG;
    Box3 ob = to_box(out_box), xb = to_box(x_box), yb = to_box(y_box);
    Box3 r = intersect(intersect(ob, xb), yb);
    if (bempty(r)) return PB_OK;
    k_axpby<<<grid_for(bvol(r), 256), 256, 0, (cudaStream_t)stream>>>(out, ob, x, xb, y, yb, region_of(r), a, b);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_reduce_async_f64(int op, const double* data, pb_box box, pb_box region, double* result_dev, void* stream)
{
    if (!data || !result_dev || op < 0 || op > 5) return PB_ERR_ARG;
    Box3 b = to_box(box), r = to_box(region);
    if (bempty(b)) return PB_ERR_BOX;
    r = bempty(r) ? b : intersect(r, b);
    RedScratch* s;
    int e = red_scratch(&s);
    if (e != PB_OK) return e;
    Region rg;
    if (bempty(r)) { rg.lo[0] = rg.lo[1] = rg.lo[2] = 0; rg.n[0] = rg.n[1] = rg.n[2] = 0; }
    else rg = region_of(r);
    long long total = bempty(r) ? 0 : bvol(r);
    int grid = (int)((total + kRedThreads - 1) / kRedThreads);
    if (grid > kRedBlocks) grid = kRedBlocks;
    if (grid < 1) grid = 1;
    k_reduce<<<grid, kRedThreads, 0, (cudaStream_t)stream>>>(op, data, b, rg, s->partials, s->ticket, result_dev);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_reduce_f64(int op, const double* data, pb_box box, pb_box region, double* result, void* stream)
{
    if (!result) return PB_ERR_ARG;
    RedScratch* s;
    int e = red_scratch(&s);
    if (e != PB_OK) return e;
    e = pb_reduce_async_f64(op, data, box, region, s->result, stream);
    if (e != PB_OK) return e;
    cudaStream_t st = (cudaStream_t)stream;
    PB_CUDA(cudaMemcpyAsync(result, s->result, sizeof(double), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
    return PB_OK;
}

int pb_interp_constant_f64(int ratio, const double* src, pb_box src_box, double* dst, pb_box dst_box, int overwrite,
                           double scale, void* stream)
{
    if (!src || !dst || ratio < 1) return PB_ERR_ARG;
    Box3 sb = to_box(src_box), db = to_box(dst_box);
    if (bempty(sb) || bempty(db)) return PB_ERR_BOX;
    Box3 rb;
    for (int d = 0; d < 3; d++) { rb.lo[d] = sb.lo[d] * ratio; rb.hi[d] = sb.hi[d] * ratio + ratio - 1; }
    rb = intersect(rb, db);
    if (bempty(rb)) return PB_OK;
    // InterpStencil::apply's final stage is "S = scale*Shift::Zeros()", folded like hostApply
    k_interp_const<<<grid_for(bvol(rb), 256), 256, 0, (cudaStream_t)stream>>>(ratio, src, sb, dst, db, region_of(rb),
                                                                            overwrite, scale);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

} // extern "C"
