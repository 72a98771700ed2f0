// Batched phase kernels of the serving engine: one launch runs one V-cycle phase (a smoothing
// sweep, a restriction, a prolongation, the FP64 residual pass or the fused update) for every
// in-flight solve at once. A phase is a list of items (one grid level of one solve each) in device
// memory; the kernels are persistent (grid fixed, work read from the list), so a captured CUDA
// graph of a whole cycle stays valid while solves come and go.
//
// Each item's work units (cells) start at a multiple of kSvUnit in the phase's index space, so a
// block-wide chunk of kSvUnit units lies in one item: the block finds it with one binary search.
// The per-cell arithmetic is the single-solve solver's (same helpers, same order), so a solve's
// result does not depend on what else is in the batch.
#pragma once
#include "pb_mg_kernels.cuh"

namespace pb {

constexpr int kSvUnit = 256;       // threads per block = units per chunk
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
    int units;             // work units of this item
    long long unit0;       // first unit (multiple of kSvUnit)
};

struct SvPhaseHeader {
    long long count;       // items
    long long total;       // units spanned (multiple of kSvUnit)
};

// item holding the chunk that starts at unit w (items sorted by unit0)
__device__ __forceinline__ int sv_find(const SvItem* items, int count, long long w)
{
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].unit0 <= w) lo = mid;
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
                                                      const SvPhaseHeader* __restrict__ hdr, double* norms)
{
    const int count = (int)hdr->count;
    const long long total = hdr->total;
    for (long long w0 = (long long)blockIdx.x * kSvUnit; w0 < total; w0 += (long long)gridDim.x * kSvUnit) {
        const SvItem& it = items[sv_find(items, count, w0)];
        const int i = (int)(w0 - it.unit0) + threadIdx.x;
        double m = 0.0;
        if (i < it.units) {
            const int n = it.k.n, sx = it.k.sx;
            int x, y, z;
            sv_cell(i, n, x, y, z);
            if constexpr (OP == SV_RELAX || OP == SV_UPDATE) {
                const long long Sy = sx, Sz = (long long)sx * (n + 2);
                const long long g = grown_index<float>(n, sx, x, y, z);
                float acc = 0.f;
#pragma unroll
                for (int j = 0; j < ShapeLap7::NT; j++) {
                    const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
                    acc = dadd(acc, dmul(it.c.c[j], it.in[g + o]));
                }
                const float v = relax_value(it.k, acc, it.in[g], it.rhs[i], it.alpha);
                if constexpr (OP == SV_RELAX) {
                    store_periodic(it.out, n, sx, x, y, z, v);
                } else {
                    const long long gd = grown_index<double>(n, it.sxd, x, y, z);
                    store_periodic(it.u64, n, it.sxd, x, y, z, dadd(it.u64[gd], (double)v));
                }
            } else if constexpr (OP == SV_RELAX_FIRST) {
                store_periodic(it.out, n, sx, x, y, z, relax_value(it.k, 0.f, 0.f, it.rhs[i], it.alpha));
            } else if constexpr (OP == SV_RESTRICT) {
                // unit = coarse cell of the (n/2)^3 level below; 8 fine residuals in Box([0,1]^3) order
                const int nc = n / 2;
                sv_cell(i, nc, x, y, z);
                const long long Sy = sx, Sz = (long long)sx * (n + 2);
                float acc = 0.f;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
                    const int fi = fx + n * (fy + n * fz);
                    const float r = fine_residual(it.in, grown_index<float>(n, sx, fx, fy, fz), Sy, Sz, it.rhs[fi],
                                                  it.alpha, it.k.helm, it.c, it.beta);
                    acc = dadd(acc, dmul(0.125f, r));
                }
                it.out[i] = acc;
            } else if constexpr (OP == SV_PROLONG) {
                const float d = it.delta[grown_index<float>(n / 2, it.sxc, x / 2, y / 2, z / 2)];
                const long long g = grown_index<float>(n, sx, x, y, z);
                store_periodic(it.in, n, sx, x, y, z, dadd(it.in[g], dmul(1.f, d)));
            } else if constexpr (OP == SV_K1) {
                // FP64 residual of u64, its max-norm, the FP32 right-hand side and the first FP32 sweep
                const int sxd = it.sxd;
                const long long Sy = sxd, Sz = (long long)sxd * (n + 2);
                const long long g = grown_index<double>(n, sxd, x, y, z);
                double res;
                float al = 0.f;
                if (!it.k.helm) {
                    res = dadd(0.0, it.f64[i]);
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
                    res = dsub(it.f64[i], dsub(dmul(it.alpha64, it.u64[g]), dmul(it.beta64, lp)));
                    al = __double2float_rn(it.alpha64);
                }
                m = upd_abs(0.0, res);
                const float r32 = __double2float_rn(res);
                it.out[i] = r32;   // the level's rho
                store_periodic(it.in, n, sx, x, y, z, relax_value(it.k, 0.f, 0.f, r32, al));
            }
        }
        if constexpr (OP == SV_K1) {
            // the chunk lies in one item: one max per warp, one atomic per warp
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(0xffffffffu, m, o);
                m = (m < w) ? w : m;
            }
            if ((threadIdx.x & 31) == 0 && m > 0.0) atomic_max_nonneg(norms + it.slot, m);
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
