// FAS multigrid with the 4th-order flux-form Laplacian (C ABI: pb_fas_*).
//
// Reference counterparts (paths within the reference project):
//   LevelMultigridSolver::solve / resnorm ....... include/utils/implem/Proto_LevelMultigridSolverImplem.H:85-159
//   MGLevel::relax / coarseForce / fineCorrect / vCycle ..................... same file :261-433
//   BoxOp::operator() (flux divergence, fluxScale) include/base/implem/Proto_BoxOpImplem.H:125-172
//   BoxOp_Laplace::flux (DiffCellToFace(d, Lo, 4)) examples/_common/BoxOp_Laplace.H:22-27
//   averageDown .................................. include/base/implem/Proto_LevelBoxDataImplem.H:993-1038
// The reference evaluates the operator patch by patch through four temporaries (three face-flux
// BoxData and a divergence) after an exchange; here every level is one periodic box with a
// two-cell ghost layer and one kernel per step evaluates, per cell, the same operations in the same
// order (face gradients with |=, the divergence with +=, the sum, the flux scale -1), so the
// residual history and the solution are bitwise the reference's. Kernels that write a state also
// write its periodic ghost images.
#include <cmath>
#include <vector>

#include "pb_internal.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

PB_DEFINE_ERROR_READER(read_error_fas)

constexpr int kFasGhost = 2;

struct FasCoef {
    double g[4];     // DiffCellToFace(d, Lo, 4) * 1/dx, offsets -2, -1, 0, +1 along d
    double cp, c0;   // divergence 1.0*Shift(+e) - 1.0*Shift(0), * 1/dx
};

// grown index of valid cell (x, y, z) with ghost 2: edge n, extent S = n + 4
__device__ __forceinline__ long long fas_index(int S, int x, int y, int z)
{
    return (x + kFasGhost) + (long long)S * ((y + kFasGhost) + (long long)S * (z + kFasGhost));
}

// op(u) at cell i (grown index), 4th-order flux-form Laplacian with flux scale -1
__device__ __forceinline__ double fas_op(const double* u, long long i, int S, const FasCoef& k)
{
    double div = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long long e = d == 0 ? 1 : (d == 1 ? (long long)S : (long long)S * S);
        double fp = 0.0, fm = 0.0;
#pragma unroll
        for (int t = 0; t < 4; t++) fp = dadd(fp, dmul(k.g[t], u[i + e + (t - 2) * e]));
#pragma unroll
        for (int t = 0; t < 4; t++) fm = dadd(fm, dmul(k.g[t], u[i + (t - 2) * e]));
        div = dadd(div, dmul(k.cp, fp));
        div = dadd(div, dmul(k.c0, fm));
    }
    return dmul(dadd(0.0, div), -1.0);
}

// writes v to valid cell (x,y,z) and every ghost cell (width 2) that is a periodic image of it
__device__ void fas_store(double* u, int n, int x, int y, int z, double v)
{
    const int S = n + 2 * kFasGhost;
    for (int kz = -2; kz <= 2; kz++) {
        const int zz = z + kz * n;
        if (zz < -kFasGhost || zz >= n + kFasGhost) continue;
        for (int ky = -2; ky <= 2; ky++) {
            const int yy = y + ky * n;
            if (yy < -kFasGhost || yy >= n + kFasGhost) continue;
            for (int kx = -2; kx <= 2; kx++) {
                const int xx = x + kx * n;
                if (xx < -kFasGhost || xx >= n + kFasGhost) continue;
                u[fas_index(S, xx, yy, zz)] = v;
            }
        }
    }
}

__device__ __forceinline__ void fas_cell(long long i, int n, int& x, int& y, int& z)
{
    x = (int)(i % n);
    const long long q = i / n;
    y = (int)(q % n);
    z = (int)(q / n);
}

#define FAS_LOOP(total)                                                                                        \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (total);                          \
         i += (long long)gridDim.x * blockDim.x)

// Jacobi sweep: out = u + (-lambda) * (op(u) + f), periodic images included
__global__ void __launch_bounds__(256) k_fas_relax(const double* __restrict__ u, double* out,
                                                   const double* __restrict__ f, int n, FasCoef k, double neg_lambda)
{
    const int S = n + 2 * kFasGhost;
    FAS_LOOP((long long)n * n * n)
    {
        int x, y, z;
        fas_cell(i, n, x, y, z);
        const long long g = fas_index(S, x, y, z);
        const double res = dadd(fas_op(u, g, S, k), f[i]);
        fas_store(out, n, x, y, z, dadd(u[g], dmul(neg_lambda, res)));
    }
}

// coarse state = AvgDown(u) (with images) and its copy c0
__global__ void __launch_bounds__(256) k_fas_average(const double* __restrict__ u, double* uc, double* c0, int nf)
{
    const int nc = nf / 2, S = nf + 2 * kFasGhost;
    FAS_LOOP((long long)nc * nc * nc)
    {
        int x, y, z;
        fas_cell(i, nc, x, y, z);
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 8; c++)
            acc = dadd(acc, dmul(0.125, u[fas_index(S, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2))]));
        fas_store(uc, nc, x, y, z, acc);
        c0[i] = acc;
    }
}

// coarse force, first part: fc = AvgDown(op(u) + f)
__global__ void __launch_bounds__(256) k_fas_restrict(const double* __restrict__ u, const double* __restrict__ f,
                                                      double* fc, int nf, FasCoef k)
{
    const int nc = nf / 2, S = nf + 2 * kFasGhost;
    FAS_LOOP((long long)nc * nc * nc)
    {
        int x, y, z;
        fas_cell(i, nc, x, y, z);
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int fx = 2 * x + (c & 1), fy = 2 * y + ((c >> 1) & 1), fz = 2 * z + (c >> 2);
            const double res = dadd(fas_op(u, fas_index(S, fx, fy, fz), S, k), f[fx + (long long)nf * (fy + (long long)nf * fz)]);
            acc = dadd(acc, dmul(0.125, res));
        }
        fc[i] = acc;
    }
}

// coarse force, second part: fc -= op_c(uc)
__global__ void __launch_bounds__(256) k_fas_force(const double* __restrict__ uc, double* fc, int nc, FasCoef k)
{
    const int S = nc + 2 * kFasGhost;
    FAS_LOOP((long long)nc * nc * nc)
    {
        int x, y, z;
        fas_cell(i, nc, x, y, z);
        fc[i] = dsub(fc[i], fas_op(uc, fas_index(S, x, y, z), S, k));
    }
}

// fine correction: c0 = -(c0 - uc) on the coarse grid, then u += 1.0 * c0(p/2) (images included)
__global__ void __launch_bounds__(256) k_fas_delta(double* c0, const double* __restrict__ uc, int nc)
{
    const int S = nc + 2 * kFasGhost;
    FAS_LOOP((long long)nc * nc * nc)
    {
        int x, y, z;
        fas_cell(i, nc, x, y, z);
        c0[i] = dmul(dsub(c0[i], uc[fas_index(S, x, y, z)]), -1.0);
    }
}
__global__ void __launch_bounds__(256) k_fas_correct(double* u, const double* __restrict__ c0, int nf)
{
    const int nc = nf / 2, S = nf + 2 * kFasGhost;
    FAS_LOOP((long long)nf * nf * nf)
    {
        int x, y, z;
        fas_cell(i, nf, x, y, z);
        const double d = c0[x / 2 + (long long)nc * (y / 2 + (long long)nc * (z / 2))];
        fas_store(u, nf, x, y, z, dadd(u[fas_index(S, x, y, z)], dmul(1.0, d)));
    }
}

// max |op(u) + f|  (Reduction<Abs>: NaN ignored)
__global__ void __launch_bounds__(256) k_fas_resnorm(const double* __restrict__ u, const double* __restrict__ f, int n,
                                                     FasCoef k, double* result)
{
    const int S = n + 2 * kFasGhost;
    double m = 0.0;
    FAS_LOOP((long long)n * n * n)
    {
        int x, y, z;
        fas_cell(i, n, x, y, z);
        m = upd_abs(m, dadd(fas_op(u, fas_index(S, x, y, z), S, k), f[i]));
    }
    block_max_atomic(m, result);
}

__global__ void __launch_bounds__(256) k_fas_pack(const double* __restrict__ src, double* u, int n)
{
    FAS_LOOP((long long)n * n * n)
    {
        int x, y, z;
        fas_cell(i, n, x, y, z);
        fas_store(u, n, x, y, z, src[i]);
    }
}
__global__ void __launch_bounds__(256) k_fas_unpack(const double* __restrict__ u, double* dst, int n)
{
    const int S = n + 2 * kFasGhost;
    FAS_LOOP((long long)n * n * n)
    {
        int x, y, z;
        fas_cell(i, n, x, y, z);
        dst[i] = u[fas_index(S, x, y, z)];
    }
}

struct FasLevel {
    int n;
    double dx;
    FasCoef k;
    double neg_lambda;
    double* u[2] = {nullptr, nullptr};   // ping-pong state, grown
    int cur = 0;
    double* f = nullptr;                  // n^3
    double* c0 = nullptr;                 // n^3: copy of the averaged-down state (coarse levels)
};

static FasCoef fas_coefs(double dx)
{
    static const double base[4] = {1.0, -15.0, 15.0, -1.0};
    const double s = 1.0 / dx;
    FasCoef k;
    for (int t = 0; t < 4; t++) {
        const double c = base[t] * (1.0 / 12.0);
        k.g[t] = (s != 1.0) ? c * s : c;
    }
    k.cp = (s != 1.0) ? 1.0 * s : 1.0;
    k.c0 = (s != 1.0) ? -1.0 * s : -1.0;
    return k;
}

} // namespace pb

struct pb_fas {
    std::vector<pb::FasLevel> lv;   // 0 = coarsest
    double* d_res = nullptr;
    double* h_res = nullptr;
    int num_pre = 6, num_post = 6, num_bottom = 10;
};

using namespace pb;

static int fas_relax(pb_fas* m, int l, int sweeps, cudaStream_t st)
{
    FasLevel& L = m->lv[l];
    const long long n3 = (long long)L.n * L.n * L.n;
    for (int s = 0; s < sweeps; s++) {
        k_fas_relax<<<grid_for(n3, 256), 256, 0, st>>>(L.u[L.cur], L.u[1 - L.cur], L.f, L.n, L.k, L.neg_lambda);
        PB_LAUNCH_CHECK();
        L.cur = 1 - L.cur;
    }
    return PB_OK;
}

static int fas_vcycle(pb_fas* m, int l, cudaStream_t st)
{
    if (l == 0) return fas_relax(m, l, m->num_bottom, st);
    FasLevel& L = m->lv[l];
    FasLevel& C = m->lv[l - 1];
    int e;
    if ((e = fas_relax(m, l, m->num_pre, st)) != PB_OK) return e;
    const long long nc3 = (long long)C.n * C.n * C.n, n3 = (long long)L.n * L.n * L.n;
    C.cur = 0;
    k_fas_average<<<grid_for(nc3, 256), 256, 0, st>>>(L.u[L.cur], C.u[0], C.c0, L.n);
    PB_LAUNCH_CHECK();
    k_fas_restrict<<<grid_for(nc3, 256), 256, 0, st>>>(L.u[L.cur], L.f, C.f, L.n, L.k);
    PB_LAUNCH_CHECK();
    k_fas_force<<<grid_for(nc3, 256), 256, 0, st>>>(C.u[0], C.f, C.n, C.k);
    PB_LAUNCH_CHECK();
    if ((e = fas_vcycle(m, l - 1, st)) != PB_OK) return e;
    k_fas_delta<<<grid_for(nc3, 256), 256, 0, st>>>(C.c0, C.u[C.cur], C.n);
    PB_LAUNCH_CHECK();
    k_fas_correct<<<grid_for(n3, 256), 256, 0, st>>>(L.u[L.cur], C.c0, L.n);
    PB_LAUNCH_CHECK();
    return fas_relax(m, l, m->num_post, st);
}

static int fas_resnorm(pb_fas* m, cudaStream_t st, double* out)
{
    FasLevel& T = m->lv.back();
    PB_CUDA(cudaMemsetAsync(m->d_res, 0, sizeof(double), st));
    k_fas_resnorm<<<grid_for((long long)T.n * T.n * T.n, 256), 256, 0, st>>>(T.u[T.cur], T.f, T.n, T.k, m->d_res);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaMemcpyAsync(m->h_res, m->d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
    *out = *m->h_res;
    return PB_OK;
}

static void fas_free(pb_fas* m)
{
    for (auto& L : m->lv) {
        cudaFree(L.u[0]);
        cudaFree(L.u[1]);
        cudaFree(L.f);
        cudaFree(L.c0);
    }
    cudaFree(m->d_res);
    cudaFreeHost(m->h_res);
    delete m;
}

extern "C" {

int pb_fas_create(int n, int num_levels, pb_fas** out)
{
    if (!out || n < 1 || num_levels < 1 || num_levels > 20) return PB_ERR_ARG;
    if ((n >> (num_levels - 1)) < 1 || ((n >> (num_levels - 1)) << (num_levels - 1)) != n) return PB_ERR_ARG;
    pb_fas* m = new (std::nothrow) pb_fas;
    if (!m) return PB_ERR_NOMEM;
    m->lv.resize(num_levels);
    bool ok = true;
    for (int l = 0; l < num_levels && ok; l++) {
        FasLevel& L = m->lv[l];
        L.n = n >> (num_levels - 1 - l);
        L.dx = (double)(1 << (num_levels - 1 - l)) / (double)n;
        L.k = fas_coefs(L.dx);
        // lambda = 0.5 / spectralRadius, spectralRadius = (2*DIM) / dx^2
        L.neg_lambda = -(0.5 / ((2.0 * 3) / std::pow(L.dx, 2)));
        const size_t g = sizeof(double) * (size_t)(L.n + 4) * (L.n + 4) * (L.n + 4), c = sizeof(double) * (size_t)L.n * L.n * L.n;
        ok = cudaMalloc(&L.u[0], g) == cudaSuccess && cudaMalloc(&L.u[1], g) == cudaSuccess &&
             cudaMalloc(&L.f, c) == cudaSuccess && cudaMalloc(&L.c0, c) == cudaSuccess &&
             cudaMemset(L.u[0], 0, g) == cudaSuccess && cudaMemset(L.u[1], 0, g) == cudaSuccess;
    }
    if (ok) ok = cudaMalloc(&m->d_res, sizeof(double)) == cudaSuccess && cudaMallocHost(&m->h_res, sizeof(double)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        fas_free(m);
        return PB_ERR_NOMEM;
    }
    *out = m;
    return PB_OK;
}

int pb_fas_destroy(pb_fas* m)
{
    if (m) fas_free(m);
    return PB_OK;
}

int pb_fas_solve(pb_fas* m, const double* force, double* phi, int max_iter, double tol, int* iters, double* hist,
                 void* stream)
{
    if (!m || !force || !phi || max_iter < 0) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    FasLevel& T = m->lv.back();
    const long long n3 = (long long)T.n * T.n * T.n;
    T.cur = 0;
    PB_CUDA(cudaMemcpyAsync(T.f, force, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
    k_fas_pack<<<grid_for(n3, 256), 256, 0, st>>>(phi, T.u[0], T.n);
    PB_LAUNCH_CHECK();
    double r0, r;
    int e;
    if ((e = fas_resnorm(m, st, &r0)) != PB_OK) return e;
    if (hist) hist[0] = r0;
    int it = 0;
    while (it < max_iter) {
        if ((e = fas_vcycle(m, (int)m->lv.size() - 1, st)) != PB_OK) return e;
        if ((e = fas_resnorm(m, st, &r)) != PB_OK) return e;
        ++it;
        if (hist) hist[it] = r;
        if (r < tol * r0) break;
    }
    k_fas_unpack<<<grid_for(n3, 256), 256, 0, st>>>(T.u[T.cur], phi, T.n);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaStreamSynchronize(st));
    if (read_error_fas() > 0) return PB_ERR_DEVICE;
    if (iters) *iters = it;
    return PB_OK;
}

} // extern "C"
