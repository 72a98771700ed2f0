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
#include <cstring>
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

// the ghost cells (width 2) that are periodic images of valid cell (x, y, z), the cell itself excluded
__device__ __noinline__ void fas_images(double* u, int n, int x, int y, int z, double v)
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
                if (xx < -kFasGhost || xx >= n + kFasGhost || (kx | ky | kz) == 0) continue;
                u[fas_index(S, xx, yy, zz)] = v;
            }
        }
    }
}

// the same for edges n >= 4, where a cell has at most one image per axis (7 in all, near a corner)
__device__ __noinline__ void fas_images_n4(double* u, int n, int x, int y, int z, double v)
{
    const int S = n + 2 * kFasGhost;
    const int ix = x < 2 ? n : (x >= n - 2 ? -n : 0);
    const int iy = y < 2 ? n : (y >= n - 2 ? -n : 0);
    const int iz = z < 2 ? n : (z >= n - 2 ? -n : 0);
#pragma unroll
    for (int c = 1; c < 8; c++) {
        const int dx = (c & 1) ? ix : 0, dy = (c & 2) ? iy : 0, dz = (c & 4) ? iz : 0;
        if (((c & 1) && !ix) || ((c & 2) && !iy) || ((c & 4) && !iz)) continue;
        u[fas_index(S, x + dx, y + dy, z + dz)] = v;
    }
}

// one face flux of DiffCellToFace(d, Lo, 4): the four cells below-below .. above of the face
__device__ __forceinline__ double fas_flux(const FasCoef& k, double a, double b, double c, double d)
{
    double f = 0.0;
    f = dadd(f, dmul(k.g[0], a));
    f = dadd(f, dmul(k.g[1], b));
    f = dadd(f, dmul(k.g[2], c));
    return dadd(f, dmul(k.g[3], d));
}

// The Jacobi sweep of k_fas_relax on large levels, two adjacent x cells per thread: a CTA owns a
// (2 kFasTX) x kFasTY column of cells and a chunk of zd planes; per plane it stages the column's
// tile with its 2-cell x/y halo (ghost cells are valid: every writer stores the periodic images)
// into a ring of shared-memory planes with 16-byte cp.async copies, kFasLead planes ahead; z
// neighbours come from a register window fed from the ring's centre column. A face flux shared by
// two cells is computed once (the x face between the pair; the z face between consecutive planes):
// it is the same four products summed in the same order either way, so every cell's value is
// bitwise fas_op's. Periodic images are written for cells within 2 of a face.
constexpr int kFasTX = 16, kFasTY = 16, kFasThreads = kFasTX * kFasTY;
constexpr int kFasBX = 2 * kFasTX + 4, kFasBY = kFasTY + 4, kFasPlane = kFasBX * kFasBY;
constexpr int kFasLead = 2 + 3, kFasRing = kFasLead + 1;

__global__ void __launch_bounds__(kFasThreads) k_fas_relax_pair(const double* __restrict__ u, double* out,
                                                                const double* __restrict__ f, int n, int zd,
                                                                FasCoef k, double neg_lambda)
{
    constexpr int R = 2, W = 5, L = kFasLead, Q = kFasRing, PM = kFasPlane, PX = kFasBX / 2;
    __shared__ __align__(16) double ring[Q * PM];
    const int S = n + 2 * kFasGhost;
    const long long S2 = (long long)S * S;
    const int x0 = blockIdx.x * 2 * kFasTX, y0 = blockIdx.y * kFasTY, z0 = blockIdx.z * zd;
    const int z1 = min(z0 + zd, n);
    const int lx = threadIdx.x % kFasTX, ly = threadIdx.x / kFasTX;
    const int x = x0 + 2 * lx, y = y0 + ly;
    const bool act = x < n && y < n;
    constexpr int kMaxLoads = (PX * kFasBY + kFasThreads - 1) / kFasThreads;
    const double* lp[kMaxLoads];
    bool lv_[kMaxLoads];
#pragma unroll
    for (int q = 0; q < kMaxLoads; q++) {
        const int i = threadIdx.x + q * kFasThreads;
        const int hx = i % PX, hy = i / PX;
        const int xx = x0 - R + 2 * hx, yy = y0 - R + hy;
        const bool xo = hx < 1 || hx > kFasTX, yo = hy < R || hy >= kFasTY + R;
        lv_[q] = i < PX * kFasBY && !(xo && yo) && xx < n + R && yy < n + R;
        lp[q] = u + (xx + kFasGhost) + (long long)S * (yy + kFasGhost) + S2 * (z0 + kFasGhost);
    }
    const uint32_t ring0 = smem_u32(ring) + 16u * threadIdx.x;
    auto stage = [&](int zz, int slot) {
        if (zz < z1) {
#pragma unroll
            for (int q = 0; q < kMaxLoads; q++)
                if (lv_[q]) {
                    cp_async16(ring0 + 8u * (slot * PM + 2 * q * kFasThreads), lp[q]);
                    lp[q] += S2;
                }
        }
        cp_async_commit();
    };
    const double* col = u + fas_index(S, act ? x : 0, act ? y : 0, 0);   // (x, y, z = 0), pair-aligned
    auto zcol = [&](int zz) -> double2 { return __ldg(reinterpret_cast<const double2*>(col + S2 * zz)); };
#pragma unroll
    for (int q = 0; q < L; q++) stage(z0 + q, q);
    double w0[W], w1[W];
    if (act) {
#pragma unroll
        for (int q = 0; q < 2 * R; q++) {
            const double2 v = zcol(z0 - R + q);
            w0[q] = v.x;
            w1[q] = v.y;
        }
    }
    double fz0 = 0.0, fz1 = 0.0;   // lower z-face flux of the current plane (carried from the one below)
    if (act) {
        fz0 = fas_flux(k, w0[0], w0[1], w0[2], w0[3]);
        fz1 = fas_flux(k, w1[0], w1[1], w1[2], w1[3]);
    }
    const int sc = (ly + R) * kFasBX + (2 * lx + R);
    const double* fp = f + (act ? x + (long long)n * (y + (long long)n * z0) : 0);
    double* op = out + fas_index(S, act ? x : 0, act ? y : 0, z0);
    const bool edge_xy = x < 2 || x + 1 >= n - 2 || y < 2 || y >= n - 2;
    int qz = 0;
    for (int z = z0; z < z1; z++) {
        double2 fv = make_double2(0.0, 0.0);
        if (act) fv = __ldg(reinterpret_cast<const double2*>(fp));
        cp_async_wait<L - R - 1>();
        __syncthreads();
        const int qn = qz == 0 ? Q - 1 : qz - 1;
        stage(z + L, qn);
        if (act) {
            int qr = qz + R;
            if (qr >= Q) qr -= Q;
            const double2 cn = z + R < z1 ? *reinterpret_cast<const double2*>(ring + qr * PM + sc) : zcol(z + R);
            w0[2 * R] = cn.x;
            w1[2 * R] = cn.y;
            const double* pl = ring + qz * PM + sc;
            const double2 xm = *reinterpret_cast<const double2*>(pl - 2);
            const double2 xc = *reinterpret_cast<const double2*>(pl);
            const double2 xq = *reinterpret_cast<const double2*>(pl + 2);
            const double2 ym2 = *reinterpret_cast<const double2*>(pl - 2 * kFasBX);
            const double2 ym1 = *reinterpret_cast<const double2*>(pl - kFasBX);
            const double2 yp1 = *reinterpret_cast<const double2*>(pl + kFasBX);
            const double2 yp2 = *reinterpret_cast<const double2*>(pl + 2 * kFasBX);
            // x faces: below cell 0, between the pair, above cell 1
            const double fxm = fas_flux(k, xm.x, xm.y, xc.x, xc.y);
            const double fxc = fas_flux(k, xm.y, xc.x, xc.y, xq.x);
            const double fxp = fas_flux(k, xc.x, xc.y, xq.x, xq.y);
            const double gz0 = fas_flux(k, w0[1], w0[2], w0[3], w0[4]);
            const double gz1 = fas_flux(k, w1[1], w1[2], w1[3], w1[4]);
            double d0 = 0.0, d1 = 0.0;
            d0 = dadd(d0, dmul(k.cp, fxc));
            d0 = dadd(d0, dmul(k.c0, fxm));
            d0 = dadd(d0, dmul(k.cp, fas_flux(k, ym1.x, xc.x, yp1.x, yp2.x)));
            d0 = dadd(d0, dmul(k.c0, fas_flux(k, ym2.x, ym1.x, xc.x, yp1.x)));
            d0 = dadd(d0, dmul(k.cp, gz0));
            d0 = dadd(d0, dmul(k.c0, fz0));
            d1 = dadd(d1, dmul(k.cp, fxp));
            d1 = dadd(d1, dmul(k.c0, fxc));
            d1 = dadd(d1, dmul(k.cp, fas_flux(k, ym1.y, xc.y, yp1.y, yp2.y)));
            d1 = dadd(d1, dmul(k.c0, fas_flux(k, ym2.y, ym1.y, xc.y, yp1.y)));
            d1 = dadd(d1, dmul(k.cp, gz1));
            d1 = dadd(d1, dmul(k.c0, fz1));
            fz0 = gz0;
            fz1 = gz1;
            const double r0 = dadd(dmul(dadd(0.0, d0), -1.0), fv.x);
            const double r1 = dadd(dmul(dadd(0.0, d1), -1.0), fv.y);
            double2 v;
            v.x = dadd(xc.x, dmul(neg_lambda, r0));
            v.y = dadd(xc.y, dmul(neg_lambda, r1));
            *reinterpret_cast<double2*>(op) = v;
            if (edge_xy || z < 2 || z >= n - 2) {
                fas_images_n4(out, n, x, y, z, v.x);
                fas_images_n4(out, n, x + 1, y, z, v.y);
            }
#pragma unroll
            for (int q = 0; q < 2 * R; q++) {
                w0[q] = w0[q + 1];
                w1[q] = w1[q + 1];
            }
        }
        op += S2;
        fp += (long long)n * n;
        qz = qz == Q - 1 ? 0 : qz + 1;
    }
    cp_async_wait<0>();
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

// ---- the levels of edge <= kFasCoarseEdge in one CTA ------------------------------------------
// The same per-cell operations as the kernels above, in the same order (sweeps, averaging,
// coarse force, recursion, correction), each phase a block-stride loop followed by a barrier;
// the state stays in the levels' own (L2-resident) buffers. One launch replaces about thirty
// launch-bound ones; a 16^3 level already costs more FP64 work than one SM does quickly, so it
// keeps its own launches.
constexpr int kFasCoarseEdge = 8, kFasCoarseMax = 8, kFasCoarseThreads = 512;

struct FasCoarseLevel {
    int n;
    FasCoef k;
    double neg_lambda;
    double* u[2];
    double* f;
    double* c0;
};
struct FasCoarseArgs {
    FasCoarseLevel lv[kFasCoarseMax];   // 0 = coarsest
    int top;                            // index of the entry level
    int num_pre, num_post, num_bottom;
};

#define FAS_BLOCK_LOOP(total) for (long long i = threadIdx.x; i < (total); i += blockDim.x)

__device__ void fas_blk_relax(const FasCoarseLevel& L, int from, int sweeps)
{
    const int n = L.n, S = n + 2 * kFasGhost;
    const long long n3 = (long long)n * n * n;
    int c = from;
    for (int s = 0; s < sweeps; s++) {
        const double* u = L.u[c];
        double* out = L.u[1 - c];
        FAS_BLOCK_LOOP(n3)
        {
            int x, y, z;
            fas_cell(i, n, x, y, z);
            const long long g = fas_index(S, x, y, z);
            const double res = dadd(fas_op(u, g, S, L.k), L.f[i]);
            fas_store(out, n, x, y, z, dadd(u[g], dmul(L.neg_lambda, res)));
        }
        __syncthreads();
        c = 1 - c;
    }
}

__global__ void __launch_bounds__(kFasCoarseThreads) k_fas_coarse_cycle(FasCoarseArgs a)
{
    // Every level is entered with its state in buffer 0 (the entry level by its parent, the others
    // by the averaging below), so the buffer holding a level's state is fixed by the sweep counts:
    // after the pre-sweeps (and through the correction) pre & 1; at the end post-sweeps included,
    // (pre + post) & 1; the coarsest level's after its sweeps, bottom & 1.
    const int c_pre = a.num_pre & 1, c_end = (a.num_pre + a.num_post) & 1, c_bot = a.num_bottom & 1;
    // down: pre-sweeps, coarse state and force
    for (int l = a.top; l >= 1; l--) {
        const FasCoarseLevel& L = a.lv[l];
        const FasCoarseLevel& C = a.lv[l - 1];
        fas_blk_relax(L, 0, a.num_pre);
        const int nf = L.n, nc = C.n, Sf = nf + 2 * kFasGhost;
        const long long nc3 = (long long)nc * nc * nc;
        const double* u = L.u[c_pre];
        FAS_BLOCK_LOOP(nc3)
        {   // k_fas_average
            int x, y, z;
            fas_cell(i, nc, x, y, z);
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < 8; c++)
                acc = dadd(acc, dmul(0.125, u[fas_index(Sf, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2))]));
            fas_store(C.u[0], nc, x, y, z, acc);
            C.c0[i] = acc;
        }
        FAS_BLOCK_LOOP(nc3)
        {   // k_fas_restrict
            int x, y, z;
            fas_cell(i, nc, x, y, z);
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const int fx = 2 * x + (c & 1), fy = 2 * y + ((c >> 1) & 1), fz = 2 * z + (c >> 2);
                const double res = dadd(fas_op(u, fas_index(Sf, fx, fy, fz), Sf, L.k),
                                        L.f[fx + (long long)nf * (fy + (long long)nf * fz)]);
                acc = dadd(acc, dmul(0.125, res));
            }
            C.f[i] = acc;
        }
        __syncthreads();
        const int Sc = nc + 2 * kFasGhost;
        FAS_BLOCK_LOOP(nc3)
        {   // k_fas_force
            int x, y, z;
            fas_cell(i, nc, x, y, z);
            C.f[i] = dsub(C.f[i], fas_op(C.u[0], fas_index(Sc, x, y, z), Sc, C.k));
        }
        __syncthreads();
    }
    fas_blk_relax(a.lv[0], 0, a.num_bottom);
    // up: correction from the level below, post-sweeps
    for (int l = 1; l <= a.top; l++) {
        const FasCoarseLevel& L = a.lv[l];
        const FasCoarseLevel& C = a.lv[l - 1];
        const int nf = L.n, nc = C.n, Sc = nc + 2 * kFasGhost, Sf = nf + 2 * kFasGhost;
        const long long nc3 = (long long)nc * nc * nc, nf3 = (long long)nf * nf * nf;
        FAS_BLOCK_LOOP(nc3)
        {   // k_fas_delta
            int x, y, z;
            fas_cell(i, nc, x, y, z);
            C.c0[i] = dmul(dsub(C.c0[i], C.u[l - 1 == 0 ? c_bot : c_end][fas_index(Sc, x, y, z)]), -1.0);
        }
        __syncthreads();
        double* u = L.u[c_pre];
        FAS_BLOCK_LOOP(nf3)
        {   // k_fas_correct
            int x, y, z;
            fas_cell(i, nf, x, y, z);
            const double d = C.c0[x / 2 + (long long)nc * (y / 2 + (long long)nc * (z / 2))];
            fas_store(u, nf, x, y, z, dadd(u[fas_index(Sf, x, y, z)], dmul(1.0, d)));
        }
        __syncthreads();
        fas_blk_relax(L, c_pre, a.num_post);
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

// BoxOp<BoxOp_Laplace>::operator() on a box: out = ((0 + div) * flux_scale) [* scale], per cell the
// operations of fas_op with the field's own strides (state on box sb, out on box ob, range rb).
__global__ void __launch_bounds__(256) k_boxop_laplace(const double* __restrict__ u, Box3 sb, double* out, Box3 ob,
                                                       Box3 rb, FasCoef k, double flux_scale, double scale,
                                                       int apply_scale)
{
    const long long nx = bsize(rb, 0), ny = bsize(rb, 1), total = bvol(rb);
    const long long Sx = bsize(sb, 0), Sxy = Sx * bsize(sb, 1);
    const long long Ox = bsize(ob, 0), Oxy = Ox * bsize(ob, 1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int x = rb.lo[0] + (int)(i % nx), y = rb.lo[1] + (int)((i / nx) % ny), z = rb.lo[2] + (int)(i / (nx * ny));
        const long long c = (x - sb.lo[0]) + Sx * (y - sb.lo[1]) + Sxy * (z - sb.lo[2]);
        double div = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const long long e = d == 0 ? 1 : (d == 1 ? Sx : Sxy);
            double fp = 0.0, fm = 0.0;
#pragma unroll
            for (int t = 0; t < 4; t++) fp = dadd(fp, dmul(k.g[t], u[c + e + (t - 2) * e]));
#pragma unroll
            for (int t = 0; t < 4; t++) fm = dadd(fm, dmul(k.g[t], u[c + (t - 2) * e]));
            div = dadd(div, dmul(k.cp, fp));
            div = dadd(div, dmul(k.c0, fm));
        }
        double v = dmul(dadd(0.0, div), flux_scale);
        if (apply_scale) v = dmul(v, scale);
        out[(x - ob.lo[0]) + Ox * (y - ob.lo[1]) + Oxy * (z - ob.lo[2])] = v;
    }
}

} // namespace pb

struct pb_fas {
    std::vector<pb::FasLevel> lv;   // 0 = coarsest
    double* d_res = nullptr;
    double* h_res = nullptr;
    int num_pre = 6, num_post = 6, num_bottom = 10;
    // the V-cycle plus the residual norm, captured once per parity of the finest level's buffer
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_cur[2] = {0, 0};           // the finest level's buffer after the captured cycle
    cudaStream_t graph_stream = nullptr;
};

using namespace pb;

// levels of edge >= kFasPairMin (even) sweep with the staged two-cells-per-thread kernel; smaller
// ones have too few (x, y) columns to fill the GPU with z-streaming CTAs
constexpr int kFasPairMin = 128;

static int fas_relax(pb_fas* m, int l, int sweeps, cudaStream_t st)
{
    FasLevel& L = m->lv[l];
    const long long n3 = (long long)L.n * L.n * L.n;
    const bool pair = L.n >= kFasPairMin && L.n % 2 == 0;
    dim3 grid;
    int zd = 32;
    if (pair) {
        const int nbx = (L.n + 2 * kFasTX - 1) / (2 * kFasTX), nby = (L.n + kFasTY - 1) / kFasTY;
        // z chunks shallow enough for about six waves of the 3 CTAs an SM holds (tail under ~15 %)
        const long long want = 18LL * cached_sm_count();
        while (zd > 4 && (long long)nbx * nby * ((L.n + zd - 1) / zd) < want) zd /= 2;
        grid = dim3(nbx, nby, (L.n + zd - 1) / zd);
    }
    for (int s = 0; s < sweeps; s++) {
        if (pair)
            k_fas_relax_pair<<<grid, kFasThreads, 0, st>>>(L.u[L.cur], L.u[1 - L.cur], L.f, L.n, zd, L.k, L.neg_lambda);
        else
            k_fas_relax<<<grid_for(n3, 256), 256, 0, st>>>(L.u[L.cur], L.u[1 - L.cur], L.f, L.n, L.k, L.neg_lambda);
        PB_LAUNCH_CHECK();
        L.cur = 1 - L.cur;
    }
    return PB_OK;
}

// every level of edge <= kFasCoarseEdge (l and below) in one single-CTA launch; level l's state
// starts at buffer 0 (its parent has just averaged into it) and ends at the parity of its sweeps
static int fas_coarse(pb_fas* m, int l, cudaStream_t st)
{
    FasCoarseArgs a;
    memset(&a, 0, sizeof(a));
    for (int q = 0; q <= l; q++) {
        const FasLevel& L = m->lv[q];
        a.lv[q] = FasCoarseLevel{L.n, L.k, L.neg_lambda, {L.u[0], L.u[1]}, L.f, L.c0};
    }
    a.top = l;
    a.num_pre = m->num_pre;
    a.num_post = m->num_post;
    a.num_bottom = m->num_bottom;
    k_fas_coarse_cycle<<<1, kFasCoarseThreads, 0, st>>>(a);
    PB_LAUNCH_CHECK();
    FasLevel& T = m->lv[l];
    T.cur = l == 0 ? (T.cur + m->num_bottom) & 1 : (T.cur + m->num_pre + m->num_post) & 1;
    return PB_OK;
}

static int fas_vcycle(pb_fas* m, int l, cudaStream_t st)
{
    if (m->lv[l].n <= kFasCoarseEdge && l < kFasCoarseMax && l < (int)m->lv.size() - 1) return fas_coarse(m, l, st);
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

// max |op(u) + f| on the finest level into the pinned host word (stream ordered, no wait)
static int fas_enqueue_resnorm(pb_fas* m, cudaStream_t st)
{
    FasLevel& T = m->lv.back();
    PB_CUDA(cudaMemsetAsync(m->d_res, 0, sizeof(double), st));
    k_fas_resnorm<<<grid_for((long long)T.n * T.n * T.n, 256), 256, 0, st>>>(T.u[T.cur], T.f, T.n, T.k, m->d_res);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaMemcpyAsync(m->h_res, m->d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    return PB_OK;
}

static int fas_resnorm(pb_fas* m, cudaStream_t st, double* out)
{
    const int e = fas_enqueue_resnorm(m, st);
    if (e != PB_OK) return e;
    PB_CUDA(cudaStreamSynchronize(st));
    *out = *m->h_res;
    return PB_OK;
}

static int fas_cycle_and_norm(pb_fas* m, cudaStream_t st)
{
    const int e = fas_vcycle(m, (int)m->lv.size() - 1, st);
    return e != PB_OK ? e : fas_enqueue_resnorm(m, st);
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
    for (int p = 0; p < 2; p++)
        if (m->graph[p]) cudaGraphExecDestroy(m->graph[p]);
    if (m->graph_stream) cudaStreamDestroy(m->graph_stream);
    delete m;
}

extern "C" {

int pb_boxop_laplace_f64(const double* state, pb_box state_box, double* out, pb_box out_box, pb_box range, double dx,
                         double flux_scale, double scale, void* stream)
{
    if (!state || !out || !(dx > 0)) return PB_ERR_ARG;
    const Box3 sb = to_box(state_box), ob = to_box(out_box);
    Box3 rb = to_box(range);
    if (bempty(sb) || bempty(ob)) return PB_ERR_BOX;
    if (bempty(rb)) rb = ob;
    if (!contains_box(ob, rb)) return PB_ERR_BOX;
    Box3 need = rb;
    for (int d = 0; d < 3; d++) {
        need.lo[d] -= kFasGhost;      // the face fluxes reach two cells down and two up
        need.hi[d] += kFasGhost;
    }
    if (!contains_box(sb, need)) return PB_ERR_GHOST;
    const long long total = bvol(rb);
    k_boxop_laplace<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(state, sb, out, ob, rb, fas_coefs(dx),
                                                                            flux_scale, scale, scale != 1.0);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

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
        const int par = T.cur;
        if (!m->graph[par]) {
            if (!m->graph_stream) PB_CUDA(cudaStreamCreateWithFlags(&m->graph_stream, cudaStreamNonBlocking));
            cudaGraph_t g;
            PB_CUDA(cudaStreamBeginCapture(m->graph_stream, cudaStreamCaptureModeThreadLocal));
            e = fas_cycle_and_norm(m, m->graph_stream);
            cudaError_t ce = cudaStreamEndCapture(m->graph_stream, &g);
            if (e != PB_OK) {
                if (ce == cudaSuccess) cudaGraphDestroy(g);
                return e;
            }
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            ce = cudaGraphInstantiate(&m->graph[par], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) { m->graph[par] = nullptr; set_cuda_error(ce); return PB_ERR_CUDA; }
            m->graph_cur[par] = T.cur;   // capture recorded the buffer flips without running them
            T.cur = par;
        }
        PB_CUDA(cudaGraphLaunch(m->graph[par], st));
        T.cur = m->graph_cur[par];
        PB_CUDA(cudaStreamSynchronize(st));
        r = *m->h_res;
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
