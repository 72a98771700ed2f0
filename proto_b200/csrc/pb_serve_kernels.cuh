// Batched phase kernels of the serving engine: one launch runs one V-cycle phase (a smoothing
// sweep, a restriction, a prolongation, the FP64 residual pass or the fused update) for every
// in-flight solve at once. A phase is a list of items (one grid level of one solve each) in device
// memory; the kernels are persistent (grid fixed, work read from the list), so a captured CUDA
// graph of a whole cycle stays valid while solves come and go.
//
// Work units are grid rows (one (y, z) pair; a restriction's rows are coarse rows). A block takes
// kSvRows consecutive rows, one warp per row, lanes striding along x (coalesced). Each item's rows
// start at a multiple of kSvRows, so a chunk lies in one item: the block finds it with one binary
// search over the phase's compact array of first rows.
// The per-cell arithmetic is the single-solve solver's (same helpers, same order), so a solve's
// result does not depend on what else is in the batch.
#pragma once
#include "pb_mg_kernels.cuh"

namespace pb {

constexpr int kSvUnit = 256;       // threads per block
constexpr int kSvRows = kSvUnit / 32;   // rows per chunk (one warp each)
constexpr int kSvMaxSolves = 256;  // solves in flight at most

struct SvItem {
    float* in;             // relax: source phi; restrict: fine phi; prolong: fine phi (updated in place);
                           // K1: the level's phi[1] (receives the first sweep)
    float* out;            // relax: destination phi; restrict: coarse rho; K1: the level's rho
    const float* rhs;      // this level's rho (n^3)
    const float* delta;    // prolong: coarse phi
    double* u64;           // K1 / update: FP64 solution (grown, pitch sxd)
    const double* f64;     // K1: FP64 right-hand side (n^3)
    RelaxCoef<float> k;    // n, sx, helm and the smoother's scalars of this level
    Coefs<float> c;        // relax: L(., omega/6) | L(., 1/h^2); restrict: L(., -1/h^2) | L(., 1/h^2)
    Coefs<double> c64;     // K1: L(., -1/h^2) | L(., 1/h^2)
    float alpha, beta;     // Helmholtz scalars
    double alpha64, beta64;
    int sxc;               // prolong: coarse pitch
    int sxd;               // K1 / update: pitch of u64
    int slot;              // solve slot (norms)
    int units;             // rows of this item
    long long unit0;       // first row (multiple of kSvRows)
};

struct SvPhaseHeader {
    long long count;       // items
    long long total;       // rows spanned (multiple of kSvRows)
};

// item holding the chunk that starts at row w (first rows ascending, in a compact array)
__device__ __forceinline__ int sv_find(const long long* __restrict__ unit0, int count, long long w)
{
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(unit0 + mid) <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

enum SvOp { SV_RELAX = 0, SV_RELAX_FIRST = 1, SV_RESTRICT = 2, SV_PROLONG = 3, SV_K1 = 4, SV_UPDATE = 5 };

__device__ __forceinline__ void sv_cell(int i, int n, int& x, int& y, int& z)
{
    x = i % n;
    y = (i / n) % n;
    z = i / (n * n);
}

template <int OP>
__global__ void __launch_bounds__(kSvUnit) k_sv_phase(const SvItem* __restrict__ items,
                                                      const long long* __restrict__ unit0,
                                                      const SvPhaseHeader* __restrict__ hdr, double* norms)
{
    const int count = (int)hdr->count;
    const long long total = hdr->total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (long long w0 = (long long)blockIdx.x * kSvRows; w0 < total; w0 += (long long)gridDim.x * kSvRows) {
        const SvItem& it = items[sv_find(unit0, count, w0)];
        const int row = (int)(w0 - it.unit0) + warp;
        double m = 0.0;
        if (row < it.units) {
            const int n = it.k.n, sx = it.k.sx;
            if constexpr (OP == SV_RESTRICT) {
                // a row of coarse cells of the (n/2)^3 level below; 8 fine residuals each, Box([0,1]^3) order
                const int nc = n / 2;
                const int y = row % nc, z = row / nc;
                const long long Sy = sx, Sz = (long long)sx * (n + 2);
                float* out = it.out + (long long)row * nc;
                for (int x = lane; x < nc; x += 32) {
                    float acc = 0.f;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
                        const int fi = fx + n * (fy + n * fz);
                        const float r = fine_residual<float>(it.in, grown_index<float>(n, sx, fx, fy, fz), Sy, Sz,
                                                             it.rhs[fi], it.alpha, it.k.helm, it.c, it.beta);
                        acc = dadd(acc, dmul(0.125f, r));
                    }
                    out[x] = acc;
                }
            } else {
                const int y = row % n, z = row / n;
                const int ey = edge_code(y, n), ez = edge_code(z, n);
                const long long g0 = grown_index<float>(n, sx, 0, y, z);   // valid cell x = 0 of the row
                const long long i0 = (long long)row * n;                    // its n^3 index
                if constexpr (OP == SV_RELAX || OP == SV_UPDATE) {
                    const long long Sy = sx, Sz = (long long)sx * (n + 2);
                    const long long gd0 = OP == SV_UPDATE ? grown_index<double>(n, it.sxd, 0, y, z) : 0;
                    for (int x = lane; x < n; x += 32) {
                        const long long g = g0 + x;
                        float acc = 0.f;
#pragma unroll
                        for (int j = 0; j < ShapeLap7::NT; j++) {
                            const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
                            acc = dadd(acc, dmul(it.c.c[j], it.in[g + o]));
                        }
                        const float v = relax_value(it.k, acc, it.in[g], it.rhs[i0 + x], it.alpha);
                        if constexpr (OP == SV_RELAX) {
                            store_with_images(it.out, n, sx, it.out + g, edge_code(x, n), ey, ez, v);
                        } else {
                            double* q = it.u64 + gd0 + x;
                            store_with_images(it.u64, n, it.sxd, q, edge_code(x, n), ey, ez, dadd(*q, (double)v));
                        }
                    }
                } else if constexpr (OP == SV_RELAX_FIRST) {
                    for (int x = lane; x < n; x += 32)
                        store_with_images(it.out, n, sx, it.out + g0 + x, edge_code(x, n), ey, ez,
                                          relax_value(it.k, 0.f, 0.f, it.rhs[i0 + x], it.alpha));
                } else if constexpr (OP == SV_PROLONG) {
                    const float* d = it.delta + grown_index<float>(n / 2, it.sxc, 0, y / 2, z / 2);
                    for (int x = lane; x < n; x += 32) {
                        float* q = it.in + g0 + x;
                        store_with_images(it.in, n, sx, q, edge_code(x, n), ey, ez, dadd(*q, dmul(1.f, d[x / 2])));
                    }
                } else if constexpr (OP == SV_K1) {
                    // FP64 residual of u64, its max-norm, the FP32 right-hand side and the first FP32 sweep
                    const int sxd = it.sxd;
                    const long long Sy = sxd, Sz = (long long)sxd * (n + 2);
                    const long long gd0 = grown_index<double>(n, sxd, 0, y, z);
                    const float al = it.k.helm ? __double2float_rn(it.alpha64) : 0.f;
                    for (int x = lane; x < n; x += 32) {
                        const long long g = gd0 + x;
                        double res;
                        if (!it.k.helm) {
                            res = dadd(0.0, it.f64[i0 + x]);
#pragma unroll
                            for (int j = 0; j < ShapeLap7::NT; j++) {
                                const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
                                res = dadd(res, dmul(it.c64.c[j], it.u64[g + o]));
                            }
                        } else {
                            double lp = 0.0;
#pragma unroll
                            for (int j = 0; j < ShapeLap7::NT; j++) {
                                const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
                                lp = dadd(lp, dmul(it.c64.c[j], it.u64[g + o]));
                            }
                            res = dsub(it.f64[i0 + x], dsub(dmul(it.alpha64, it.u64[g]), dmul(it.beta64, lp)));
                        }
                        m = upd_abs(m, res);
                        const float r32 = __double2float_rn(res);
                        it.out[i0 + x] = r32;   // the level's rho
                        store_with_images(it.in, n, sx, it.in + g0 + x, edge_code(x, n), ey, ez,
                                          relax_value(it.k, 0.f, 0.f, r32, al));
                    }
                }
            }
        }
        if constexpr (OP == SV_K1) {
            // a warp's row lies in one item: one max per warp, one atomic per warp
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(0xffffffffu, m, o);
                m = (m < w) ? w : m;
            }
            if (lane == 0 && m > 0.0 && row < it.units) atomic_max_nonneg(norms + it.slot, m);
        }
    }
}

// u64 (grown, periodic) -> dst (n^3), one launch per solve being retired
static __global__ void __launch_bounds__(256) k_sv_pack_out(const double* __restrict__ u, double* dst, int n, int sxd)
{
    const long long total = (long long)n * n * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        sv_cell((int)i, n, x, y, z);
        dst[i] = u[grown_index<double>(n, sxd, x, y, z)];
    }
}

// constant fill (alpha fields of the coarse levels)
static __global__ void __launch_bounds__(256) k_sv_fill(float* p, long long n, float v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

} // namespace pb
