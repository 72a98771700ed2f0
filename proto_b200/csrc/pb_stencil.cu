// Stencil objects and Stencil::apply on the device (C ABI: pb_stencil_*).
//
// Replaces the reference's DEVICE branch of Stencil::protoApply
// (include/base/implem/Proto_StencilImplem.H:844-895 in the reference project), whose kernel runs
// one thread per point with coefficients read from global memory. Here:
//   * the seven- and thirteen-point Laplacians (in the exact insertion order the reference's
//     StencilLib produces) run on the TMA-staged z-streaming kernel of pb_star.cuh, or on its
//     one-thread-per-point variant for small or unaligned boxes;
//   * every other stencil (any ratios, destination shift, up to kMaxTerms terms) runs on a
//     table kernel with the coefficients and linearised offsets in kernel parameters.
// All FP64 results equal Stencil::hostApply bit for bit (term order, scale folded into the
// coefficients when scale != 1, no FMA).
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "pb_internal.cuh"
#include "pb_star.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

PB_DEFINE_ERROR_READER(read_error_stencil)

// The bounded wait of the pipelined kernels, made to expire on purpose: one thread waits on an
// mbarrier whose phase never completes (nothing arrives and no copy is in flight), gives up after
// `tries` polls through the same mbar_wait_limited every kernel uses, and records whether the wait
// reported the timeout; the wait also sets the device error flag that pb_device_check reads.
static __device__ int g_wait_expired = 0;
static __global__ void k_wait_expiry(uint32_t tries)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) g_wait_expired = mbar_wait_limited(&bar, 0, tries) ? 0 : 1;
}

static thread_local int t_last_cuda = 0;
void set_cuda_error(cudaError_t e) { t_last_cuda = (int)e; }

// ---- TMA tensor-map encoding through the driver entry point (no -lcuda link needed) ----------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn g_encode = nullptr;
static std::once_flag g_encode_once;

static void load_encode()
{
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_encode = reinterpret_cast<EncodeTiledFn>(fn);
    cudaGetLastError();
}

bool tma_available()
{
    std::call_once(g_encode_once, load_encode);
    return g_encode != nullptr;
}

int encode_tmap_3d(CUtensorMap* map, const void* base, int esize, long long Sx, long long Sy, long long Sz, int boxX,
                   int boxY, int boxZ)
{
    if (!tma_available()) return PB_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return PB_ERR_ALIGN;
    if ((Sx * esize) % 16 != 0) return PB_ERR_ALIGN;
    if (boxX > 256 || boxY > 256 || boxZ > 256 || (boxX * esize) % 16 != 0) return PB_ERR_ALIGN;
    cuuint64_t gdim[3] = {(cuuint64_t)Sx, (cuuint64_t)Sy, (cuuint64_t)Sz};
    cuuint64_t gstr[2] = {(cuuint64_t)(Sx * esize), (cuuint64_t)(Sx * Sy * esize)};
    cuuint32_t box[3] = {(cuuint32_t)boxX, (cuuint32_t)boxY, (cuuint32_t)boxZ};
    cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMapDataType dt = esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = g_encode(map, dt, 3, const_cast<void*>(base), gdim, gstr, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? PB_OK : PB_ERR_ALIGN;
}

// ---- generic table kernel ---------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_table(const T* __restrict__ src, T* dst, const TableArgs<T> a)
{
    const long long nx = a.ib.hi[0] - a.ib.lo[0] + 1, ny = a.ib.hi[1] - a.ib.lo[1] + 1,
                    nz = a.ib.hi[2] - a.ib.lo[2] + 1;
    const long long total = nx * ny * nz;
    const long long sSx = a.sb.hi[0] - a.sb.lo[0] + 1, sSy = a.sb.hi[1] - a.sb.lo[1] + 1;
    const long long dSx = a.db.hi[0] - a.db.lo[0] + 1, dSy = a.db.hi[1] - a.db.lo[1] + 1;
    const long long svol = sSx * sSy * (a.sb.hi[2] - a.sb.lo[2] + 1);
    const long long dvol = dSx * dSy * (a.db.hi[2] - a.db.lo[2] + 1);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int p[3];
        p[0] = a.ib.lo[0] + (int)(i % nx);
        long long r = i / nx;
        p[1] = a.ib.lo[1] + (int)(r % ny);
        p[2] = a.ib.lo[2] + (int)(r / ny);
        int dp[3];
        bool inside = true;
        for (int d = 0; d < 3; d++) {
            dp[d] = p[d] * a.dr[d] + a.ds[d];
            inside &= (dp[d] >= a.db.lo[d]) && (dp[d] <= a.db.hi[d]);
        }
        if (!inside) continue;
        const long long di = (dp[0] - a.db.lo[0]) + dSx * ((dp[1] - a.db.lo[1]) + dSy * (long long)(dp[2] - a.db.lo[2]));
        const long long si = (p[0] * a.sr[0] - a.sb.lo[0]) +
                             sSx * ((p[1] * a.sr[1] - a.sb.lo[1]) + sSy * (long long)(p[2] * a.sr[2] - a.sb.lo[2]));
        for (int c = 0; c < a.ncomp; c++) {
            const T* s = src + c * svol;
            T* o = dst + c * dvol;
            T acc = a.init_zero ? T(0) : o[di];
            for (int j = 0; j < a.n; j++) acc = dadd(acc, dmul(a.c[j], __ldg(s + si + a.off[j])));
            o[di] = acc;
        }
    }
}

// ---- host-side stencil object -----------------------------------------------------------------
} // namespace pb

struct pb_stencil {
    std::vector<double> coefs;
    std::vector<int> offs;   // n x 3
    int sr[3], dr[3], ds[3];
    int spanLo[3], spanHi[3];
    int shape;               // 0 table, 1 Lap7, 2 Lap13
};

namespace pb {

template <class S>
static bool matches_shape(const pb_stencil* s)
{
    if ((int)s->coefs.size() != S::NT) return false;
    for (int d = 0; d < 3; d++)
        if (s->sr[d] != 1 || s->dr[d] != 1 || s->ds[d] != 0) return false;
    for (int j = 0; j < S::NT; j++)
        for (int d = 0; d < 3; d++)
            if (s->offs[3 * j + d] != S::off(j, d)) return false;
    return true;
}

// scale folded into the coefficients as Stencil::hostApply does (Proto_StencilImplem.H:771-779)
template <typename T>
static inline T fold(double c, T scale)
{
    return scale != T(1) ? (T)c * scale : (T)c;
}

int cached_sm_count()
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

int grid_for(long long total, int threads)
{
    long long b = (total + threads - 1) / threads;
    long long cap = (long long)cached_sm_count() * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

int stencil_coefs(const pb_stencil* s, double* c, int cap)
{
    int n = (int)s->coefs.size();
    for (int j = 0; j < n && j < cap; j++) c[j] = s->coefs[j];
    return n;
}

static StarTune g_default_tune;
StarTune& default_star_tune() { return g_default_tune; }

} // namespace pb

// Launch-shape knobs of the star kernels (used by the autotuner and by profiling sweeps):
// mode 0 auto / 1 TMA only / 2 simple only; zc z-chunk (0 heuristic); (ty, yb, xv) CTA tile height,
// rows per consumer thread and adjacent x points per consumer thread (xv 0: one point per thread
// for Stencil::apply, two for the multigrid sweeps).
extern "C" int pb_star_tune_set(int mode, int zc, int ty, int yb, int xv, long long min_tma_points)
{
    const bool shape_ok = (ty == 8 && yb == 1 && xv == 1) || (ty == 8 && yb == 2 && xv >= 0 && xv <= 2) ||
                          (ty == 4 && yb == 2 && xv == 2);
    if (mode < 0 || mode > 2 || zc < 0 || !shape_ok) return PB_ERR_ARG;
    pb::StarTune& t = pb::default_star_tune();
    t.mode = mode;
    t.zc = zc;
    t.ty = ty;
    t.yb = yb;
    t.xv = xv;
    if (min_tma_points >= 0) t.min_tma_points = min_tma_points;
    return PB_OK;
}

extern "C" int pb_star_tune_ring(int nst, int aux_smem)
{
    if (nst != 0 && (nst < 3 || nst > 16)) return PB_ERR_ARG;
    if (aux_smem != 0 && aux_smem != 1) return PB_ERR_ARG;
    pb::StarTune& t = pb::default_star_tune();
    t.nst = nst;
    t.aux_smem = aux_smem;
    return PB_OK;
}

namespace pb {

// ---- apply dispatch ---------------------------------------------------------------------------
static inline OutMap out_map(const Box3& ib, const Box3& db)
{
    OutMap m;
    m.dx = ib.lo[0] - db.lo[0];
    m.dy = ib.lo[1] - db.lo[1];
    m.dz = ib.lo[2] - db.lo[2];
    m.Dx = bsize(db, 0);
    m.Dxy = bsize(db, 0) * bsize(db, 1);
    return m;
}

// Validate / infer the index box; returns PB_OK or an error status.
static int resolve_box(const pb_stencil* s, const Box3& sb, const Box3& db, pb_box box, Box3* out)
{
    Box3 ib = to_box(box);
    if (bempty(ib)) {
        // indexDomain(dst) & indexRange(src) (Proto_StencilImplem.H:324-346)
        Box3 r, d;
        for (int k = 0; k < 3; k++) {
            r.lo[k] = sb.lo[k] - s->spanLo[k];
            r.hi[k] = sb.hi[k] - s->spanHi[k];
            d.lo[k] = db.lo[k] - s->ds[k];
            d.hi[k] = db.hi[k] - s->ds[k];
        }
        ib = intersect(taper_coarsen(r, s->sr), taper_coarsen(d, s->dr));
    }
    // the source must hold every point the terms read
    if (!bempty(ib)) {
        Box3 need;
        for (int k = 0; k < 3; k++) {
            need.lo[k] = ib.lo[k] * s->sr[k] + s->spanLo[k];
            need.hi[k] = ib.hi[k] * s->sr[k] + s->spanHi[k];
        }
        if (!contains_box(sb, need)) return PB_ERR_GHOST;
    }
    *out = ib;
    return PB_OK;
}

template <typename T>
static int apply_impl(const pb_stencil* s, const T* src, pb_box src_box, T* dst, pb_box dst_box, pb_box box,
                      int ncomp, int init_to_zero, T scale, cudaStream_t st)
{
    if (!s || !src || !dst || ncomp < 1) return PB_ERR_ARG;
    Box3 sb = to_box(src_box), db = to_box(dst_box), ib;
    if (bempty(sb) || bempty(db)) return PB_ERR_BOX;
    int e = resolve_box(s, sb, db, box, &ib);
    if (e != PB_OK) return e;
    if (bempty(ib) || s->coefs.empty()) return PB_OK;
    if (scale == T(0)) {
        // the reference zeroes the destination for "|=" and does nothing else
        if (!init_to_zero) return PB_OK;
        TableArgs<T> a;
        memset(&a, 0, sizeof(a));
        a.n = 0;
        a.ncomp = ncomp;
        a.init_zero = 1;
        a.sb = sb; a.db = db; a.ib = ib;
        for (int k = 0; k < 3; k++) { a.sr[k] = s->sr[k]; a.dr[k] = s->dr[k]; a.ds[k] = s->ds[k]; }
        k_table<T><<<grid_for(bvol(ib), 256), 256, 0, st>>>(src, dst, a);
        PB_LAUNCH_CHECK();
        return PB_OK;
    }
    const long long svol = bvol(sb), dvol = bvol(db);
    if (s->shape == 1 || s->shape == 2) {
        // star kernels: destination ratio 1, no shift -> clip to the destination box
        Box3 cib = intersect(ib, db);
        if (bempty(cib)) return PB_OK;
        Coefs<T> cf;
        for (int j = 0; j < (int)s->coefs.size(); j++) cf.c[j] = fold<T>(s->coefs[j], scale);
        for (int c = 0; c < ncomp; c++) {
            EpiStore<T> epi;
            epi.dst = dst + c * dvol;
            epi.m = out_map(cib, db);
            epi.accumulate = !init_to_zero;
            int r = (s->shape == 1) ? launch_star<ShapeLap7>(src + c * svol, sb, cib, cf, epi, st, default_star_tune())
                                    : launch_star<ShapeLap13>(src + c * svol, sb, cib, cf, epi, st, default_star_tune());
            if (r != PB_OK) return r;
        }
        return PB_OK;
    }
    int n = (int)s->coefs.size();
    if (n > kMaxTerms) return PB_ERR_UNSUPPORTED;
    TableArgs<T> a;
    a.n = n;
    a.ncomp = ncomp;
    a.init_zero = init_to_zero ? 1 : 0;
    a.sb = sb; a.db = db; a.ib = ib;
    for (int k = 0; k < 3; k++) { a.sr[k] = s->sr[k]; a.dr[k] = s->dr[k]; a.ds[k] = s->ds[k]; }
    const long long sSx = bsize(sb, 0), sSxy = bsize(sb, 0) * bsize(sb, 1);
    for (int j = 0; j < n; j++) {
        a.c[j] = fold<T>(s->coefs[j], scale);
        a.off[j] = s->offs[3 * j] + sSx * s->offs[3 * j + 1] + sSxy * s->offs[3 * j + 2];
    }
    k_table<T><<<grid_for(bvol(ib), 256), 256, 0, st>>>(src, dst, a);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

} // namespace pb

using namespace pb;

extern "C" {

const char* pb_status_string(int s)
{
    switch (s) {
        case PB_OK: return "ok";
        case PB_ERR_ARG: return "invalid argument";
        case PB_ERR_BOX: return "invalid box";
        case PB_ERR_CUDA: return "CUDA runtime error";
        case PB_ERR_ALIGN: return "alignment requirement not met";
        case PB_ERR_NOMEM: return "out of memory";
        case PB_ERR_UNSUPPORTED: return "unsupported request";
        case PB_ERR_BUDGET: return "memory budget exceeded";
        case PB_ERR_DEVICE: return "device-side error flagged";
        case PB_ERR_GHOST: return "source box does not cover the stencil footprint";
    }
    return "unknown status";
}

int pb_last_cuda_error(void) { return t_last_cuda; }

const char* pb_version(void) { return "proto_b200 1.0 sm_100a"; }

int pb_debug_wait_expiry(unsigned int tries, int* expired, void* stream)
{
    if (!expired || tries == 0 || tries > kMaxWaitTries) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_wait_expiry<<<1, 32, 0, st>>>(tries);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaStreamSynchronize(st));
    PB_CUDA(cudaMemcpyFromSymbol(expired, g_wait_expired, sizeof(int)));
    return PB_OK;
}

int pb_device_check(void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    PB_CUDA(cudaStreamSynchronize(st));
    int a = read_error_stencil(), b = read_error_mg(), c = read_error_serve(), d = read_error_fas();
    if (a < 0 || b < 0 || c < 0 || d < 0) return PB_ERR_CUDA;
    return (a || b || c || d) ? PB_ERR_DEVICE : PB_OK;
}

int pb_stencil_create(const double* coefs, const int* offsets, int nterms, const int src_ratio[3],
                      const int dst_ratio[3], const int dst_shift[3], pb_stencil** out)
{
    if (!out || nterms < 0 || (nterms > 0 && (!coefs || !offsets))) return PB_ERR_ARG;
    pb_stencil* s = new (std::nothrow) pb_stencil;
    if (!s) return PB_ERR_NOMEM;
    s->coefs.assign(coefs, coefs + nterms);
    s->offs.assign(offsets, offsets + 3 * nterms);
    for (int d = 0; d < 3; d++) {
        s->sr[d] = src_ratio ? src_ratio[d] : 1;
        s->dr[d] = dst_ratio ? dst_ratio[d] : 1;
        s->ds[d] = dst_shift ? dst_shift[d] : 0;
        if (s->sr[d] <= 0 || s->dr[d] <= 0) { delete s; return PB_ERR_ARG; }
        s->spanLo[d] = 0;
        s->spanHi[d] = 0;
    }
    // span: Stencil::addCoef grows it with every offset (Proto_StencilImplem.H:238-276)
    for (int j = 0; j < nterms; j++)
        for (int d = 0; d < 3; d++) {
            int v = offsets[3 * j + d];
            if (j == 0 || v < s->spanLo[d]) s->spanLo[d] = v;
            if (j == 0 || v > s->spanHi[d]) s->spanHi[d] = v;
        }
    s->shape = matches_shape<ShapeLap7>(s) ? 1 : matches_shape<ShapeLap13>(s) ? 2 : 0;
    *out = s;
    return PB_OK;
}

int pb_stencil_destroy(pb_stencil* s)
{
    delete s;
    return PB_OK;
}

int pb_stencil_info(const pb_stencil* s, int* nterms, pb_box* span, int* shape)
{
    if (!s) return PB_ERR_ARG;
    if (nterms) *nterms = (int)s->coefs.size();
    if (span)
        for (int d = 0; d < 3; d++) { span->lo[d] = s->spanLo[d]; span->hi[d] = s->spanHi[d]; }
    if (shape) *shape = s->shape;
    return PB_OK;
}

int pb_stencil_apply_f64(const pb_stencil* s, const double* src, pb_box src_box, double* dst, pb_box dst_box,
                         pb_box box, int ncomp, int init_to_zero, double scale, void* stream)
{
    return apply_impl<double>(s, src, src_box, dst, dst_box, box, ncomp, init_to_zero, scale, (cudaStream_t)stream);
}

int pb_stencil_apply_f32(const pb_stencil* s, const float* src, pb_box src_box, float* dst, pb_box dst_box,
                         pb_box box, int ncomp, int init_to_zero, float scale, void* stream)
{
    return apply_impl<float>(s, src, src_box, dst, dst_box, box, ncomp, init_to_zero, scale, (cudaStream_t)stream);
}

int pb_stencil_apply_fused_f64(const pb_stencil* s, int epilogue, const double* u, pb_box u_box, double* out,
                               pb_box out_box, pb_box box, double scale, double a, double b, void* stream)
{
    if (!s || !u || !out) return PB_ERR_ARG;
    if (epilogue != PB_EPI_AXPBY && epilogue != PB_EPI_EULER) return PB_ERR_ARG;
    if (s->shape != 1 && s->shape != 2) return PB_ERR_UNSUPPORTED;
    Box3 sb = to_box(u_box), db = to_box(out_box), ib;
    if (bempty(sb) || bempty(db)) return PB_ERR_BOX;
    int e = resolve_box(s, sb, db, box, &ib);
    if (e != PB_OK) return e;
    ib = intersect(ib, db);
    if (bempty(ib)) return PB_OK;
    Coefs<double> cf;
    for (int j = 0; j < (int)s->coefs.size(); j++) cf.c[j] = fold<double>(s->coefs[j], scale);
    EpiAxpby<double> epi;
    epi.dst = out;
    epi.m = out_map(ib, db);
    epi.a = a;
    epi.b = b;
    epi.euler = (epilogue == PB_EPI_EULER);
    cudaStream_t st = (cudaStream_t)stream;
    return (s->shape == 1) ? launch_star<ShapeLap7>(u, sb, ib, cf, epi, st, default_star_tune())
                           : launch_star<ShapeLap13>(u, sb, ib, cf, epi, st, default_star_tune());
}

} // extern "C"
