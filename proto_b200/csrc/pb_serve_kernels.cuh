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
    int zd;                // column-walk phases: z planes per unit (chosen per phase)
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

// The stencil phases (sweep, sweep + FP64 update, FP64 residual pass) as warp column walks: a unit
// is (row y, 32-wide x chunk, z chunk of kSvZ planes); a warp's lanes take consecutive x and walk
// z with a register window of the 7-point stencil's z taps; +-x come from neighbouring lanes
// (shuffles; the chunk's end lanes load the cell beyond, a ghost image at the box faces), +-y are
// direct loads. Terms are summed in the Laplacian's insertion order, so results are bitwise the
// row kernel's.
constexpr int kSvZ = 16;   // deepest z chunk (a phase with few units takes shallower ones)

__device__ __forceinline__ void sv_walk_units(int n, int zd, int& xc_count, int& zc_count)
{
    xc_count = (n + 31) / 32;
    zc_count = (n + zd - 1) / zd;
}

template <int OP, typename V>
__global__ void __launch_bounds__(kSvUnit) k_sv_walk(const SvItem* __restrict__ items, const long long* __restrict__ unit0,
                                                     const SvPhaseHeader* __restrict__ hdr, double* norms)
{
    const int count = (int)hdr->count;
    const long long total = hdr->total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (long long w0 = (long long)blockIdx.x * kSvRows; w0 < total; w0 += (long long)gridDim.x * kSvRows) {
        const SvItem* itp = items + sv_find(unit0, count, w0);
        const int unit = (int)(w0 - itp->unit0) + warp;
        const int units = itp->units;
        double m = 0.0;
        if (unit < units) {
            // the item's fields, once, into registers
            const RelaxCoef<float> k = itp->k;
            const int n = k.n;
            const int zd = itp->zd;
            float* const in32 = itp->in;
            float* const out32 = itp->out;
            const float* const rhs = itp->rhs;
            double* const u64 = itp->u64;
            const double* const f64 = itp->f64;
            const int sxd = itp->sxd;
            const float alpha = itp->alpha;
            const double alpha64 = itp->alpha64, beta64 = itp->beta64;
            Coefs<V> cf;
            if constexpr (OP == SV_K1) cf = itp->c64;
            else cf = itp->c;
            int XC, ZC;
            sv_walk_units(n, zd, XC, ZC);
            const int y = unit % n, xc = (unit / n) % XC, zc = unit / (n * XC);
            const int x = xc * 32 + lane;
            const bool act = x < n;
            const bool last = act && (lane == 31 || x == n - 1);
            const int z0 = zc * zd, z1 = min(z0 + zd, n);
            // source field (FP32 level for the sweeps, FP64 u for the residual pass)
            const V* src;
            int sx;
            if constexpr (OP == SV_K1) {
                src = reinterpret_cast<const V*>(u64);
                sx = sxd;
            } else {
                src = reinterpret_cast<const V*>(in32);
                sx = k.sx;
            }
            const int Sy = sx, Sz = sx * (n + 2), nn = n * n;
            const V* c = src + (long long)grown_index<V>(n, sx, act ? x : 0, y, z0);   // (x, y, z0)
            const int ey = edge_code(y, n), ex = act ? edge_code(x, n) : 0;
            int i = (act ? x : 0) + n * (y + n * z0);
            // plane z's loads are issued one plane ahead: +z, +-y, the chunk-end x neighbours and the
            // pointwise inputs (rhs; f for the residual pass; u64 for the update)
            V zm = act ? c[-Sz] : V(0), z_ = act ? c[0] : V(0);
            V zp_n = V(0), ym_n = V(0), yp_n = V(0), xme_n = V(0), xpe_n = V(0);
            float r_n = 0.f;
            double d_n = 0.0;
            auto fetch = [&](const V* cc, int ii, int zz) {
                if (!act) return;
                zp_n = cc[Sz];
                ym_n = cc[-Sy];
                yp_n = cc[Sy];
                if (lane == 0) xme_n = cc[-1];
                if (last) xpe_n = cc[1];
                if constexpr (OP == SV_K1) d_n = f64[ii];
                else r_n = rhs[ii];
                if constexpr (OP == SV_UPDATE) d_n = u64[grown_index<double>(n, sxd, x, y, zz)];
            };
            fetch(c, i, z0);
            for (int z = z0; z < z1; z++) {
                const V zp = zp_n, ym = ym_n, yp = yp_n, xme = xme_n, xpe = xpe_n;
                const float rr = r_n;
                const double dd = d_n;
                if (z + 1 < z1) fetch(c + Sz, i + nn, z + 1);
                // neighbours along x from the lanes beside (the chunk's end lanes load them)
                V xm = __shfl_up_sync(0xffffffffu, z_, 1);
                V xp = __shfl_down_sync(0xffffffffu, z_, 1);
                if (lane == 0) xm = xme;
                if (last) xp = xpe;
                if (act) {
                    const int ez = edge_code(z, n);
                    // Laplacian insertion order: 0, +x, -x, +y, -y, +z, -z
                    if constexpr (OP == SV_K1) {
                        double res;
                        float al = 0.f;
                        if (!k.helm) {
                            res = dadd(0.0, dd);
                            res = dadd(res, dmul(cf.c[0], (double)z_));
                            res = dadd(res, dmul(cf.c[1], (double)xp));
                            res = dadd(res, dmul(cf.c[2], (double)xm));
                            res = dadd(res, dmul(cf.c[3], (double)yp));
                            res = dadd(res, dmul(cf.c[4], (double)ym));
                            res = dadd(res, dmul(cf.c[5], (double)zp));
                            res = dadd(res, dmul(cf.c[6], (double)zm));
                        } else {
                            double lp = 0.0;
                            lp = dadd(lp, dmul(cf.c[0], (double)z_));
                            lp = dadd(lp, dmul(cf.c[1], (double)xp));
                            lp = dadd(lp, dmul(cf.c[2], (double)xm));
                            lp = dadd(lp, dmul(cf.c[3], (double)yp));
                            lp = dadd(lp, dmul(cf.c[4], (double)ym));
                            lp = dadd(lp, dmul(cf.c[5], (double)zp));
                            lp = dadd(lp, dmul(cf.c[6], (double)zm));
                            res = dsub(dd, dsub(dmul(alpha64, (double)z_), dmul(beta64, lp)));
                            al = __double2float_rn(alpha64);
                        }
                        m = upd_abs(m, res);
                        const float r32 = __double2float_rn(res);
                        out32[i] = r32;
                        float* q = in32 + grown_index<float>(n, k.sx, x, y, z);
                        store_with_images(in32, n, k.sx, q, ex, ey, ez, relax_value(k, 0.f, 0.f, r32, al));
                    } else {
                        float acc = 0.f;
                        acc = dadd(acc, dmul(cf.c[0], (float)z_));
                        acc = dadd(acc, dmul(cf.c[1], (float)xp));
                        acc = dadd(acc, dmul(cf.c[2], (float)xm));
                        acc = dadd(acc, dmul(cf.c[3], (float)yp));
                        acc = dadd(acc, dmul(cf.c[4], (float)ym));
                        acc = dadd(acc, dmul(cf.c[5], (float)zp));
                        acc = dadd(acc, dmul(cf.c[6], (float)zm));
                        const float v = relax_value(k, acc, (float)z_, rr, alpha);
                        if constexpr (OP == SV_RELAX) {
                            const long long g = c - src;
                            store_with_images(out32, n, sx, out32 + g, ex, ey, ez, v);
                        } else {
                            double* q = u64 + grown_index<double>(n, sxd, x, y, z);
                            store_with_images(u64, n, sxd, q, ex, ey, ez, dadd(dd, (double)v));
                        }
                    }
                }
                zm = z_;
                z_ = zp;
                c += Sz;
                i += nn;
            }
        }
        if constexpr (OP == SV_K1) {
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(0xffffffffu, m, o);
                m = (m < w) ? w : m;
            }
            if (lane == 0 && m > 0.0 && unit < units) atomic_max_nonneg(norms + itp->slot, m);
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
