// Point-Jacobi correction-scheme multigrid on periodic single-box levels (C ABI: pb_mg_*).
//
// Reference counterparts (paths within the reference project):
//   LevelMultigrid (archived 7-point solver) .. examples/_archived/LevelMultigrid/src/LevelMultigrid.cpp
//       pointRelax :90-114, coarseResidual :48-69, resnorm :71-88, fineInterp :116-131, vCycle :133-158
//   LevelMultigridSolver::vCycle / relax ....... include/utils/implem/Proto_LevelMultigridSolverImplem.H:361-433
//   averageDown / InterpStencil::Constant ..... include/base/implem/Proto_LevelBoxDataImplem.H:993-1038,
//                                               include/base/implem/Proto_InterpStencilDefs.H:1-15
// The reference runs each smoothing sweep as an exchange (one copy kernel per motion item), a
// stencil into a freshly allocated BoxData, and two more full-grid passes. Here one level is one
// periodic box with a one-cell ghost layer; every kernel that writes the solution also writes the
// periodic ghost images of the cells it owns, so no exchange pass exists, and each step is one
// fused kernel:
//   relax          : phi_new = phi + (L(phi, w) + (-lambda)*rho)           (Jacobi, out of place)
//   relax_first    : the same with phi == 0 (first sweep of a coarse correction; reads only rho)
//   resid_restrict : rho_c = AvgDown(rho + L(phi, -1/h^2))                  (8 residuals per coarse cell)
//   prolong        : phi += 1.0 * delta_c(p/2)                               (in place)
//   resnorm        : max | -rho + L(phi, 1/h^2) |                           (block max + one atomic)
// Each kernel repeats the reference's floating-point operations in the reference's order with no
// FMA, so the FP64 solver reproduces the reference CPU path's residual history bit for bit.
#include <cstring>
#include <vector>

#include "pb_internal.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

PB_DEFINE_ERROR_READER(read_error_mg)

// Writes v to the valid cell (x,y,z) of an (n+2)^3 grown periodic box and to every ghost cell
// that is a periodic image of it.
template <typename T>
__device__ __forceinline__ void store_periodic(T* out, int n, int x, int y, int z, T v)
{
    const long long S = n + 2, S2 = S * S;
    int xs[3], ys[3], zs[3];
    int nx = 1, ny = 1, nz = 1;
    xs[0] = x + 1;
    ys[0] = y + 1;
    zs[0] = z + 1;
    if (x == 0) xs[nx++] = n + 1;
    if (x == n - 1) xs[nx++] = 0;
    if (y == 0) ys[ny++] = n + 1;
    if (y == n - 1) ys[ny++] = 0;
    if (z == 0) zs[nz++] = n + 1;
    if (z == n - 1) zs[nz++] = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) out[xs[i] + S * ys[j] + S2 * zs[k]] = v;
}

template <typename T>
struct MGLevelArgs {
    const T* rhs;      // n^3
    const T* alpha;    // n^3 (Helmholtz)
    T* out;            // (n+2)^3
    int n;
    int helm;
    T neg_lambda;      // Poisson form
    T beta, omega, diagB;
};

// relax epilogue: acc = L(phi, w) (Poisson) or L(phi, 1/h^2) (Helmholtz), centre = phi
template <typename T>
struct EpiRelax {
    MGLevelArgs<T> a;
    __device__ __forceinline__ T init(int, int, int, bool) const { return T(0); }
    __device__ __forceinline__ void finish(int x, int y, int z, T acc, T c) const
    {
        const long long i = x + (long long)a.n * (y + (long long)a.n * z);
        T v;
        if (!a.helm) {
            T t = dadd(acc, dmul(a.neg_lambda, a.rhs[i]));
            v = dadd(c, t);
        } else {
            T al = a.alpha[i];
            T r = dsub(a.rhs[i], dsub(dmul(al, c), dmul(a.beta, acc)));
            v = dadd(c, ddiv(dmul(a.omega, r), dadd(al, a.diagB)));
        }
        store_periodic(a.out, a.n, x, y, z, v);
    }
    __device__ __forceinline__ void end() const {}
};

// residual max-norm epilogue: Poisson acc starts at (0 - rho) with L(phi, 1/h^2)
template <typename T>
struct EpiResnorm {
    MGLevelArgs<T> a;
    double* result;
    double m;
    __device__ __forceinline__ T init(int x, int y, int z, bool active) const
    {
        if (a.helm || !active) return T(0);
        return dsub(T(0), a.rhs[x + (long long)a.n * (y + (long long)a.n * z)]);
    }
    __device__ __forceinline__ void finish(int x, int y, int z, T acc, T c)
    {
        if (!a.helm) {
            m = upd_abs(m, (double)acc);
        } else {
            const long long i = x + (long long)a.n * (y + (long long)a.n * z);
            T r = dsub(a.rhs[i], dsub(dmul(a.alpha[i], c), dmul(a.beta, acc)));
            m = upd_abs(m, (double)r);
        }
    }
    __device__ __forceinline__ void end() { block_max_atomic(m, result); }
};

// first sweep from phi == 0 (every read of phi would return +0.0)
template <typename T>
__global__ void __launch_bounds__(256) k_relax_first(MGLevelArgs<T> a)
{
    const long long total = (long long)a.n * a.n * a.n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % a.n);
        long long q = i / a.n;
        int y = (int)(q % a.n), z = (int)(q / a.n);
        const T zero = T(0);
        T v;
        if (!a.helm) {
            T t = dadd(zero, dmul(a.neg_lambda, a.rhs[i]));
            v = dadd(zero, t);
        } else {
            T al = a.alpha[i];
            T r = dsub(a.rhs[i], dsub(dmul(al, zero), dmul(a.beta, zero)));
            v = dadd(zero, ddiv(dmul(a.omega, r), dadd(al, a.diagB)));
        }
        store_periodic(a.out, a.n, x, y, z, v);
    }
}

// coarse right-hand side: AvgDown(2) of the fine residual, children in Box([0,1]^3) order
template <typename T>
__global__ void __launch_bounds__(256) k_resid_restrict(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                        const T* __restrict__ alpha, T* rhs_c, int nf, int helm,
                                                        Coefs<T> cf, T beta)
{
    const int nc = nf / 2;
    const long long S = nf + 2, S2 = S * S;
    const long long total = (long long)nc * nc * nc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const T eighth = T(1.0 / 8);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int cx = (int)(i % nc);
        long long q = i / nc;
        int cy = (int)(q % nc), cz = (int)(q / nc);
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int fx = 2 * cx + (k & 1), fy = 2 * cy + ((k >> 1) & 1), fz = 2 * cz + (k >> 2);
            const long long fi = fx + (long long)nf * (fy + (long long)nf * fz);
            const long long gi = (fx + 1) + S * (fy + 1) + S2 * (fz + 1);
            T r;
            if (!helm) {
                r = dadd(T(0), __ldg(rhs + fi));
#pragma unroll
                for (int j = 0; j < ShapeLap7::NT; j++) {
                    const long long o = ShapeLap7::off(j, 0) + S * ShapeLap7::off(j, 1) + S2 * ShapeLap7::off(j, 2);
                    r = dadd(r, dmul(cf.c[j], __ldg(phi + gi + o)));
                }
            } else {
                T lp = T(0);
#pragma unroll
                for (int j = 0; j < ShapeLap7::NT; j++) {
                    const long long o = ShapeLap7::off(j, 0) + S * ShapeLap7::off(j, 1) + S2 * ShapeLap7::off(j, 2);
                    lp = dadd(lp, dmul(cf.c[j], __ldg(phi + gi + o)));
                }
                r = dsub(__ldg(rhs + fi), dsub(dmul(__ldg(alpha + fi), __ldg(phi + gi)), dmul(beta, lp)));
            }
            acc = dadd(acc, dmul(eighth, r));
        }
        rhs_c[i] = acc;
    }
}

// phi += 1.0 * delta_c(p/2) on the valid box, periodic images included
template <typename T>
__global__ void __launch_bounds__(256) k_prolong(T* phi, const T* __restrict__ delta_c, int nf)
{
    const int nc = nf / 2;
    const long long S = nf + 2, Sc = nc + 2;
    const long long total = (long long)nf * nf * nf;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % nf);
        long long q = i / nf;
        int y = (int)(q % nf), z = (int)(q / nf);
        T d = __ldg(delta_c + (x / 2 + 1) + Sc * (y / 2 + 1) + Sc * Sc * (z / 2 + 1));
        T v = dadd(phi[(x + 1) + S * (y + 1) + S * S * (z + 1)], dmul(T(1), d));
        store_periodic(phi, nf, x, y, z, v);
    }
}

// n^3 <-> grown (n+2)^3 with periodic ghost images
template <typename T>
__global__ void __launch_bounds__(256) k_pack_in(const T* __restrict__ src, T* out, int n)
{
    const long long total = (long long)n * n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % n);
        long long q = i / n;
        store_periodic(out, n, x, (int)(q % n), (int)(q / n), src[i]);
    }
}
template <typename T>
__global__ void __launch_bounds__(256) k_pack_out(const T* __restrict__ g, T* dst, int n)
{
    const long long total = (long long)n * n * n;
    const long long S = n + 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % n);
        long long q = i / n;
        int y = (int)(q % n), z = (int)(q / n);
        dst[i] = g[(x + 1) + S * (y + 1) + S * S * (z + 1)];
    }
}

// AvgDown(2) of a plain n^3 field (coarse-level alpha)
template <typename T>
__global__ void __launch_bounds__(256) k_avgdown_plain(const T* __restrict__ f, T* c, int nf)
{
    const int nc = nf / 2;
    const long long total = (long long)nc * nc * nc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int cx = (int)(i % nc);
        long long q = i / nc;
        int cy = (int)(q % nc), cz = (int)(q / nc);
        T acc = T(0);
        for (int k = 0; k < 8; k++) {
            int fx = 2 * cx + (k & 1), fy = 2 * cy + ((k >> 1) & 1), fz = 2 * cz + (k >> 2);
            acc = dadd(acc, dmul(T(1.0 / 8), f[fx + (long long)nf * (fy + (long long)nf * fz)]));
        }
        c[i] = acc;
    }
}

struct MGLevel {
    int n;
    double h, hsqinv;
    double* phi[2] = {nullptr, nullptr};
    double* rhs = nullptr;
    double* alpha = nullptr;
    int cur = 0;
};

} // namespace pb

struct pb_mg {
    pb_mg_params p;
    std::vector<pb::MGLevel> lv;   // index 0 = coarsest
    double* d_res = nullptr;
    double* h_res = nullptr;       // pinned
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaStream_t graph_stream = nullptr;
    int device = 0;
};

using namespace pb;

static inline double lambda_of(const pb_mg_params& p, double h) { return (p.omega * (h * h)) / 6.0; }

static int launch_relax(pb_mg* mg, int l, bool first, cudaStream_t st)
{
    MGLevel& L = mg->lv[l];
    MGLevelArgs<double> a;
    a.rhs = L.rhs;
    a.alpha = L.alpha;
    a.out = L.phi[1 - L.cur];
    a.n = L.n;
    a.helm = mg->p.form == PB_MG_HELMHOLTZ;
    a.neg_lambda = -lambda_of(mg->p, L.h);
    a.beta = mg->p.beta;
    a.omega = mg->p.omega;
    a.diagB = 6.0 * mg->p.beta * L.hsqinv;
    long long total = (long long)L.n * L.n * L.n;
    if (first) {
        k_relax_first<double><<<grid_for(total, 256), 256, 0, st>>>(a);
        PB_LAUNCH_CHECK();
    } else {
        Coefs<double> cf;
        double w = mg->p.omega / 6.0;
        double s = a.helm ? L.hsqinv : w;
        for (int j = 0; j < 7; j++) {
            double c = (j == 0) ? -6.0 : 1.0;
            cf.c[j] = (s != 1.0) ? c * s : c;
        }
        EpiRelax<double> epi;
        epi.a = a;
        Box3 sb, ib;
        for (int d = 0; d < 3; d++) { sb.lo[d] = -1; sb.hi[d] = L.n; ib.lo[d] = 0; ib.hi[d] = L.n - 1; }
        int e = launch_star<ShapeLap7>(L.phi[L.cur], sb, ib, cf, epi, st, default_star_tune());
        if (e != PB_OK) return e;
    }
    L.cur = 1 - L.cur;
    return PB_OK;
}

static int launch_resnorm(pb_mg* mg, int l, cudaStream_t st)
{
    MGLevel& L = mg->lv[l];
    PB_CUDA(cudaMemsetAsync(mg->d_res, 0, sizeof(double), st));
    EpiResnorm<double> epi;
    epi.a.rhs = L.rhs;
    epi.a.alpha = L.alpha;
    epi.a.out = nullptr;
    epi.a.n = L.n;
    epi.a.helm = mg->p.form == PB_MG_HELMHOLTZ;
    epi.a.beta = mg->p.beta;
    epi.result = mg->d_res;
    epi.m = 0.0;
    Coefs<double> cf;
    for (int j = 0; j < 7; j++) {
        double c = (j == 0) ? -6.0 : 1.0;
        cf.c[j] = (L.hsqinv != 1.0) ? c * L.hsqinv : c;
    }
    Box3 sb, ib;
    for (int d = 0; d < 3; d++) { sb.lo[d] = -1; sb.hi[d] = L.n; ib.lo[d] = 0; ib.hi[d] = L.n - 1; }
    return launch_star<ShapeLap7>(L.phi[L.cur], sb, ib, cf, epi, st, default_star_tune());
}

static int relax_sweeps(pb_mg* mg, int l, int k, bool zero_start, cudaStream_t st)
{
    for (int s = 0; s < k; s++) {
        int e = launch_relax(mg, l, zero_start && s == 0, st);
        if (e != PB_OK) return e;
    }
    if (zero_start && k == 0) {
        MGLevel& L = mg->lv[l];
        PB_CUDA(cudaMemsetAsync(L.phi[L.cur], 0, sizeof(double) * (size_t)(L.n + 2) * (L.n + 2) * (L.n + 2), st));
    }
    return PB_OK;
}

static int vcycle(pb_mg* mg, int l, bool zero_start, cudaStream_t st)
{
    MGLevel& L = mg->lv[l];
    if (zero_start) L.cur = 0;
    int e;
    if (l > 0) {
        MGLevel& C = mg->lv[l - 1];
        if ((e = relax_sweeps(mg, l, mg->p.nu1, zero_start, st)) != PB_OK) return e;
        Coefs<double> cf;
        bool helm = mg->p.form == PB_MG_HELMHOLTZ;
        double s = helm ? L.hsqinv : -L.hsqinv;
        for (int j = 0; j < 7; j++) {
            double c = (j == 0) ? -6.0 : 1.0;
            cf.c[j] = (s != 1.0) ? c * s : c;
        }
        long long nc3 = (long long)C.n * C.n * C.n;
        k_resid_restrict<double><<<grid_for(nc3, 256), 256, 0, st>>>(L.phi[L.cur], L.rhs, L.alpha, C.rhs, L.n, helm, cf,
                                                                     mg->p.beta);
        PB_LAUNCH_CHECK();
        if ((e = vcycle(mg, l - 1, true, st)) != PB_OK) return e;
        long long n3 = (long long)L.n * L.n * L.n;
        k_prolong<double><<<grid_for(n3, 256), 256, 0, st>>>(L.phi[L.cur], C.phi[C.cur], L.n);
        PB_LAUNCH_CHECK();
        return relax_sweeps(mg, l, mg->p.nu2, false, st);
    }
    return relax_sweeps(mg, l, mg->p.nu_bottom, zero_start, st);
}

static int mg_free(pb_mg* mg)
{
    for (auto& L : mg->lv) {
        cudaFree(L.phi[0]);
        cudaFree(L.phi[1]);
        cudaFree(L.alpha);
        cudaFree(L.rhs);
    }
    for (int k = 0; k < 2; k++)
        if (mg->graph[k]) cudaGraphExecDestroy(mg->graph[k]);
    if (mg->graph_stream) cudaStreamDestroy(mg->graph_stream);
    cudaFree(mg->d_res);
    cudaFreeHost(mg->h_res);
    delete mg;
    return PB_OK;
}

// One V-cycle on the finest level followed by the residual norm into h_res.
static int cycle_and_norm(pb_mg* mg, cudaStream_t st)
{
    int top = (int)mg->lv.size() - 1;
    int e = vcycle(mg, top, false, st);
    if (e != PB_OK) return e;
    if ((e = launch_resnorm(mg, top, st)) != PB_OK) return e;
    PB_CUDA(cudaMemcpyAsync(mg->h_res, mg->d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    return PB_OK;
}

static int params_ok(const pb_mg_params* p)
{
    if (!p || p->n < 1 || p->levels < 0 || p->levels > 20) return PB_ERR_ARG;
    if ((p->n >> p->levels) < 1 || ((p->n >> p->levels) << p->levels) != p->n) return PB_ERR_ARG;
    if (p->nu1 < 0 || p->nu2 < 0 || p->nu_bottom < 0 || p->max_iter < 0) return PB_ERR_ARG;
    if (p->form != PB_MG_POISSON && p->form != PB_MG_HELMHOLTZ) return PB_ERR_ARG;
    if (p->precision != PB_MG_FP64 && p->precision != PB_MG_MIXED) return PB_ERR_ARG;
    return PB_OK;
}

extern "C" {

long long pb_mg_device_bytes(const pb_mg_params* p)
{
    if (params_ok(p) != PB_OK) return -1;
    long long total = 0;
    for (int l = 0; l <= p->levels; l++) {
        long long n = p->n >> (p->levels - l);
        long long g = (n + 2) * (n + 2) * (n + 2);
        total += 2 * g * 8 + n * n * n * 8;
        if (p->form == PB_MG_HELMHOLTZ) total += n * n * n * 8;
    }
    return total + 256;
}

int pb_mg_create(const pb_mg_params* p, pb_mg** out)
{
    int e = params_ok(p);
    if (e != PB_OK) return e;
    if (!out) return PB_ERR_ARG;
    if (p->precision == PB_MG_MIXED) return PB_ERR_UNSUPPORTED;
    pb_mg* mg = new (std::nothrow) pb_mg;
    if (!mg) return PB_ERR_NOMEM;
    mg->p = *p;
    cudaGetDevice(&mg->device);
    mg->lv.resize(p->levels + 1);
    for (int l = 0; l <= p->levels; l++) {
        MGLevel& L = mg->lv[l];
        L.n = p->n >> (p->levels - l);
        L.h = (double)(1 << (p->levels - l)) / (double)p->n;
        L.hsqinv = 1. / (L.h * L.h);
        size_t g = sizeof(double) * (size_t)(L.n + 2) * (L.n + 2) * (L.n + 2);
        size_t c = sizeof(double) * (size_t)L.n * L.n * L.n;
        bool ok = cudaMalloc(&L.phi[0], g) == cudaSuccess && cudaMalloc(&L.phi[1], g) == cudaSuccess &&
                  cudaMalloc(&L.rhs, c) == cudaSuccess;
        if (ok && p->form == PB_MG_HELMHOLTZ) ok = cudaMalloc(&L.alpha, c) == cudaSuccess;
        if (ok) ok = cudaMemset(L.phi[0], 0, g) == cudaSuccess && cudaMemset(L.phi[1], 0, g) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            mg_free(mg);
            return PB_ERR_NOMEM;
        }
    }
    if (cudaMalloc(&mg->d_res, sizeof(double)) != cudaSuccess || cudaMallocHost(&mg->h_res, sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        mg_free(mg);
        return PB_ERR_NOMEM;
    }
    *out = mg;
    return PB_OK;
}

int pb_mg_destroy(pb_mg* mg)
{
    if (!mg) return PB_OK;
    return mg_free(mg);
}

int pb_mg_set_alpha(pb_mg* mg, const double* alpha, void* stream)
{
    if (!mg || !alpha) return PB_ERR_ARG;
    if (mg->p.form != PB_MG_HELMHOLTZ) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int top = (int)mg->lv.size() - 1;
    MGLevel& T = mg->lv[top];
    PB_CUDA(cudaMemcpyAsync(T.alpha, alpha, sizeof(double) * (size_t)T.n * T.n * T.n, cudaMemcpyDeviceToDevice, st));
    for (int l = top; l > 0; l--) {
        long long nc3 = (long long)mg->lv[l - 1].n * mg->lv[l - 1].n * mg->lv[l - 1].n;
        k_avgdown_plain<double><<<grid_for(nc3, 256), 256, 0, st>>>(mg->lv[l].alpha, mg->lv[l - 1].alpha, mg->lv[l].n);
        PB_LAUNCH_CHECK();
    }
    return PB_OK;
}

int pb_mg_solve(pb_mg* mg, const double* rhs, double* phi, int* iters, double* hist, void* stream)
{
    if (!mg || !rhs || !phi) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int top = (int)mg->lv.size() - 1;
    MGLevel& T = mg->lv[top];
    const long long n3 = (long long)T.n * T.n * T.n;
    PB_CUDA(cudaMemcpyAsync(T.rhs, rhs, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
    T.cur = 0;
    k_pack_in<double><<<grid_for(n3, 256), 256, 0, st>>>(phi, T.phi[0], T.n);
    PB_LAUNCH_CHECK();
    int e = launch_resnorm(mg, top, st);
    if (e != PB_OK) return e;
    PB_CUDA(cudaMemcpyAsync(mg->h_res, mg->d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
    const double r0 = *mg->h_res;
    if (hist) hist[0] = r0;
    int it = 0;
    while (it < mg->p.max_iter) {
        // replay the captured V-cycle when one exists for this buffer parity; capture otherwise
        int par = T.cur;
        if (!mg->graph[par] && it > 0) {
            if (!mg->graph_stream) PB_CUDA(cudaStreamCreateWithFlags(&mg->graph_stream, cudaStreamNonBlocking));
            cudaGraph_t g;
            PB_CUDA(cudaStreamBeginCapture(mg->graph_stream, cudaStreamCaptureModeThreadLocal));
            e = cycle_and_norm(mg, mg->graph_stream);
            cudaError_t ce = cudaStreamEndCapture(mg->graph_stream, &g);
            if (e != PB_OK) return e;
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            ce = cudaGraphInstantiate(&mg->graph[par], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            T.cur = par;   // capture recorded the parity flips without running them
            // reset the coarse levels' parity bookkeeping (they restart at zero every visit)
        }
        if (mg->graph[par]) {
            PB_CUDA(cudaGraphLaunch(mg->graph[par], st));
            // the graph flips the finest level's buffer (nu1 + nu2) times
            if ((mg->p.nu1 + mg->p.nu2) & 1) T.cur = 1 - par;
            else T.cur = par;
        } else {
            if ((e = cycle_and_norm(mg, st)) != PB_OK) return e;
        }
        PB_CUDA(cudaStreamSynchronize(st));
        const double r = *mg->h_res;
        ++it;
        if (hist) hist[it] = r;
        if (r < mg->p.tol * r0) break;
    }
    k_pack_out<double><<<grid_for(n3, 256), 256, 0, st>>>(T.phi[T.cur], phi, T.n);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaStreamSynchronize(st));
    if (iters) *iters = it;
    return PB_OK;
}

int pb_mg_relax(pb_mg* mg, int sweeps, void* stream)
{
    if (!mg || sweeps < 0) return PB_ERR_ARG;
    int top = (int)mg->lv.size() - 1;
    return relax_sweeps(mg, top, sweeps, false, (cudaStream_t)stream);
}

int pb_mg_launches_per_cycle(const pb_mg_params* p)
{
    if (params_ok(p) != PB_OK) return -1;
    // levels top..1: nu1 + nu2 sweeps, one restriction, one prolongation; bottom sweeps; one norm
    return p->levels * (p->nu1 + p->nu2 + 2) + p->nu_bottom + 1;
}

} // extern "C"
