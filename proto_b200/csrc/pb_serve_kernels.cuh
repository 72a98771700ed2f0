// Batched phase kernels of the serving engine: one launch runs one V-cycle phase (a smoothing
// sweep, a restriction, a prolongation, the FP64 residual pass or the fused update) for every
// in-flight solve at once. A phase is a list of items (one grid level of one solve each) in device
// memory; the kernels are persistent (grid fixed, work read from the list), so a captured CUDA
// graph of a whole cycle stays valid while solves come and go.
//
// Two kinds of work unit. The stencil phases (sweeps, the FP64 residual pass, the fused update)
// take a CTA per tile of a level and stage its planes through shared memory (k_sv_ring). The
// pointwise phases (restriction, prolongation, the first sweep from zero) take grid rows (one (y,
// z) pair; a restriction's rows are coarse rows): a block takes kSvRows consecutive rows, one warp
// per row, lanes striding along x (coalesced), and each item's rows start at a multiple of
// kSvRows so a chunk lies in one item. Either way a block finds its item with one binary search
// over the phase's compact array of first units.
// The per-cell arithmetic is the single-solve solver's (same helpers, same order), so a solve's
// result does not depend on what else is in the batch. The levels are FP32 in the mixed-precision
// engine (its FP64 residual pass and update work on the FP64 solution beside them) and FP64 in the
// FP64 engine, whose cycle is the FP64 solver's (the solution is the top level itself, and the
// residual norm rides on the first sweep of the next cycle).
#pragma once
#include <cfloat>
#include <math_constants.h>

#include "pb_mg_kernels.cuh"

namespace pb {

constexpr int kSvUnit = 256;       // threads per block
constexpr int kSvRows = kSvUnit / 32;   // rows per chunk (one warp each)
constexpr int kSvMaxSolves = 256;  // solves in flight at most

struct SvItem {
    // level buffers, of the engine's level type (FP32 levels of the mixed engine, FP64 levels of the
    // FP64 engine)
    void* in;              // relax / norm: source phi; restrict: fine phi; prolong: fine phi (updated
                           // in place); K1: the level's phi[1] (receives the first sweep)
    void* out;             // relax / norm: destination phi; restrict: coarse rho; K1: the level's rho
    const void* rhs;       // this level's rho (n^3)
    const void* delta;     // prolong: coarse phi
    double* u64;           // K1 / update: FP64 solution (grown, pitch sxd)
    const double* f64;     // K1: FP64 right-hand side (n^3)
    RelaxCoef<float> k;    // n, sx (the level's pitch) and the FP32 smoother's scalars of this level
    RelaxCoef<double> k64; // FP64 levels: n, sx and the smoother's scalars
    Coefs<float> c;        // relax: L(., omega/6) | L(., 1/h^2); restrict: L(., -1/h^2) | L(., 1/h^2)
    Coefs<double> c64;     // K1: L(., -1/h^2) | L(., 1/h^2); FP64 levels: as c
    double nscale;         // norm: the residual's Laplacian scale 1/h^2
    float alpha, beta;     // Helmholtz scalars of the level (FP32 levels)
    double alpha64, beta64;   // FP64 levels; K1: the top level's
    int sxc;               // prolong: coarse pitch
    int sxd;               // K1 / update: pitch of u64
    int slot;              // solve slot (norms)
    int zd;                // staged phases: z planes per unit (chosen per phase)
    int units;             // rows of this item
    long long unit0;       // first row (multiple of kSvRows)
};

// the per-level fields of an item in the level type T
template <typename T> __device__ __forceinline__ const RelaxCoef<T>& sv_k(const SvItem& it);
template <> __device__ __forceinline__ const RelaxCoef<float>& sv_k<float>(const SvItem& it) { return it.k; }
template <> __device__ __forceinline__ const RelaxCoef<double>& sv_k<double>(const SvItem& it) { return it.k64; }
template <typename T> __device__ __forceinline__ const Coefs<T>& sv_c(const SvItem& it);
template <> __device__ __forceinline__ const Coefs<float>& sv_c<float>(const SvItem& it) { return it.c; }
template <> __device__ __forceinline__ const Coefs<double>& sv_c<double>(const SvItem& it) { return it.c64; }
template <typename T> __device__ __forceinline__ T sv_alpha(const SvItem& it);
template <> __device__ __forceinline__ float sv_alpha<float>(const SvItem& it) { return it.alpha; }
template <> __device__ __forceinline__ double sv_alpha<double>(const SvItem& it) { return it.alpha64; }
template <typename T> __device__ __forceinline__ T sv_beta(const SvItem& it);
template <> __device__ __forceinline__ float sv_beta<float>(const SvItem& it) { return it.beta; }
template <> __device__ __forceinline__ double sv_beta<double>(const SvItem& it) { return it.beta64; }

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

// SV_NORM (FP64 engine): the residual max-norm of the solution fused with the next cycle's first
// sweep, as the FP64 solver's norm pass
enum SvOp { SV_RELAX = 0, SV_RELAX_FIRST = 1, SV_RESTRICT = 2, SV_PROLONG = 3, SV_K1 = 4, SV_UPDATE = 5, SV_NORM = 6 };

__device__ __forceinline__ void sv_cell(int i, int n, int& x, int& y, int& z)
{
    x = i % n;
    y = (i / n) % n;
    z = i / (n * n);
}

template <int OP, typename T>
__global__ void __launch_bounds__(kSvUnit) k_sv_phase(const SvItem* __restrict__ items,
                                                      const long long* __restrict__ unit0,
                                                      const SvPhaseHeader* __restrict__ hdr, double* norms)
{
    static_assert(OP == SV_RELAX_FIRST || OP == SV_RESTRICT || OP == SV_PROLONG, "row phases only");
    (void)norms;
    const int count = (int)hdr->count;
    const long long total = hdr->total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (long long w0 = (long long)blockIdx.x * kSvRows; w0 < total; w0 += (long long)gridDim.x * kSvRows) {
        const SvItem& it = items[sv_find(unit0, count, w0)];
        const int row = (int)(w0 - it.unit0) + warp;
        if (row < it.units) {
            const RelaxCoef<T>& kk = sv_k<T>(it);
            const Coefs<T>& cf = sv_c<T>(it);
            const T al = sv_alpha<T>(it), be = sv_beta<T>(it);
            const int n = kk.n, sx = kk.sx;
            if constexpr (OP == SV_RESTRICT) {
                // a row of coarse cells of the (n/2)^3 level below. Lanes take consecutive fine x of
                // the two fine rows and two fine planes under the row (coalesced); the taps those
                // four cells share come from registers. Each fine residual is fine_residual's
                // arithmetic (taps in the Laplacian's order); the even lane of a pair gathers its
                // neighbour's four residuals by shuffle and sums the eight children in Box([0,1]^3)
                // order.
                const int nc = n / 2;
                const int y = row % nc, z = row / nc;
                const long long Sy = sx, Sz = (long long)sx * (n + 2);
                T* out = static_cast<T*>(it.out) + (long long)row * nc;
                const T* b0 = static_cast<const T*>(it.in) + grown_index<T>(n, sx, 0, 2 * y, 2 * z);   // fine (0, 2y, 2z)
                const T* r0 = static_cast<const T*>(it.rhs) + (long long)n * (2 * y + (long long)n * (2 * z));
                for (int fx0 = 0; fx0 < n; fx0 += 32) {   // uniform over the warp (shuffles below)
                    const int fx = fx0 + lane;
                    T res[2][2] = {{T(0), T(0)}, {T(0), T(0)}};   // [dy][dz]
                    if (fx < n) {
                        const T* q = b0 + fx;
                        T c[2][2];
#pragma unroll
                        for (int dy = 0; dy < 2; dy++)
#pragma unroll
                            for (int dz = 0; dz < 2; dz++) c[dy][dz] = q[dy * Sy + dz * Sz];
#pragma unroll
                        for (int dy = 0; dy < 2; dy++)
#pragma unroll
                            for (int dz = 0; dz < 2; dz++) {
                                const T* p = q + dy * Sy + dz * Sz;
                                // 0, +x, -x, +y, -y, +z, -z
                                const T t[7] = {c[dy][dz], p[1], p[-1], dy == 0 ? c[1][dz] : p[Sy],
                                                    dy == 1 ? c[0][dz] : p[-Sy], dz == 0 ? c[dy][1] : p[Sz],
                                                    dz == 1 ? c[dy][0] : p[-Sz]};
                                const T rho = r0[fx + dy * n + (long long)dz * n * n];
                                if (!kk.helm) {
                                    T v = dadd(T(0), rho);
#pragma unroll
                                    for (int j = 0; j < 7; j++) v = dmadd(v, cf.c[j], t[j]);
                                    res[dy][dz] = v;
                                } else {
                                    T lp = T(0);
#pragma unroll
                                    for (int j = 0; j < 7; j++) lp = dmadd(lp, cf.c[j], t[j]);
                                    res[dy][dz] = dsub(rho, dsub(dmul(al, t[0]), dmul(be, lp)));
                                }
                            }
                    }
                    T odd[2][2];
#pragma unroll
                    for (int dy = 0; dy < 2; dy++)
#pragma unroll
                        for (int dz = 0; dz < 2; dz++) odd[dy][dz] = __shfl_down_sync(0xffffffffu, res[dy][dz], 1);
                    if (fx < n && (fx & 1) == 0) {
                        T acc = T(0);
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            const int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
                            acc = dmadd(acc, T(0.125), dx ? odd[dy][dz] : res[dy][dz]);
                        }
                        out[fx / 2] = acc;
                    }
                }
            } else {
                const int y = row % n, z = row / n;
                const int ey = edge_code(y, n), ez = edge_code(z, n);
                const long long g0 = grown_index<T>(n, sx, 0, y, z);   // valid cell x = 0 of the row
                const long long i0 = (long long)row * n;                    // its n^3 index
                if constexpr (OP == SV_RELAX_FIRST) {
                    T* const o = static_cast<T*>(it.out);
                    const T* const rh = static_cast<const T*>(it.rhs);
                    for (int x = lane; x < n; x += 32)
                        store_with_images(o, n, sx, o + g0 + x, edge_code(x, n), ey, ez, relax_value(kk, T(0), T(0), rh[i0 + x], al));
                } else if constexpr (OP == SV_PROLONG) {
                    const T* d = static_cast<const T*>(it.delta) + grown_index<T>(n / 2, it.sxc, 0, y / 2, z / 2);
                    T* const f = static_cast<T*>(it.in);
                    // four cells per lane in flight: their loads before their stores (a lane's stores
                    // touch only its own valid cells and their ghost images, which no load here reads)
                    for (int x0 = lane; x0 < n; x0 += 128) {
                        T v[4], dv[4];
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            const int x = x0 + 32 * k;
                            v[k] = x < n ? f[g0 + x] : T(0);
                            dv[k] = x < n ? d[x / 2] : T(0);
                        }
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            const int x = x0 + 32 * k;
                            if (x < n)
                                store_with_images(f, n, sx, f + g0 + x, edge_code(x, n), ey, ez, dadd(v[k], dmul(T(1), dv[k])));
                        }
                    }
                }
            }
        }
    }
}

// The stencil phases (sweep, FP64 residual pass, last sweep + FP64 correction) with a CTA per
// unit = (item, 32 x 16 tile of a level, chunk of zd planes); each thread owns kSvYC cells in
// consecutive rows, (x, y) .. (x, y + kSvYC - 1), so each thread carries that many independent
// accumulation chains and the block barrier and staging are shared by as many cells. Per plane the
// tile and its one-cell x/y halo are staged into a ring of shared-memory planes by 16-byte cp.async
// copies (whole 16-byte chunks of grown rows: they never cross a row's pitch, so every copy stays
// inside the level's buffer), kSvLead planes ahead of the planes being computed, one or two planes
// per block barrier; z neighbours come from register windows fed from the ring. Pointwise inputs
// (rhs, f, u64) are loaded before the barrier so their latency overlaps the wait.
// Terms are summed in the Laplacian's insertion order with the single-solve solver's epilogue
// arithmetic, so results are bitwise its.
constexpr int kSvYC = 2;                                  // cells per thread (consecutive rows)
constexpr int kSvTX = 32, kSvTY = kSvYC * (kSvUnit / 32); // 32 x 16 cells
constexpr int kSvRowStride = 36;                          // staged row: grown x0 .. x0+35 (34 used)
constexpr int kSvPlane = kSvRowStride * (kSvTY + 2);
constexpr int kSvLead = 1 + 3;   // planes staged ahead; the ring holds kSvLead + planes per barrier

__device__ __forceinline__ void sv_ring_units(int n, int zd, int& xt, int& yt, int& zt)
{
    xt = (n + kSvTX - 1) / kSvTX;
    yt = (n + kSvTY - 1) / kSvTY;
    zt = (n + zd - 1) / zd;
}

template <int OP, typename V>
__global__ void __launch_bounds__(kSvUnit, 3) k_sv_ring(const SvItem* __restrict__ items, const long long* __restrict__ unit0,
                                                     const SvPhaseHeader* __restrict__ hdr, double* norms)
{
    // planes computed per block barrier: two on FP32 levels (5 % more served solves/s), one on FP64
    // levels (two measured 1.4 % slower there)
    constexpr int PB = ((OP == SV_RELAX || OP == SV_NORM) && std::is_same<V, double>::value) ? 1 : 2;
    constexpr int L = kSvLead, Q = kSvLead + PB, PM = kSvPlane, RS = kSvRowStride;
    // level type: the mixed engine's FP32 levels (K1 and UPDATE sweep FP32 levels too), or the FP64
    // engine's levels (its sweeps and the norm pass stage FP64 planes)
    constexpr bool L64 = (OP == SV_RELAX || OP == SV_NORM) && std::is_same<V, double>::value;
    static_assert(OP != SV_NORM || L64, "the norm pass runs on FP64 levels");
    using LT = std::conditional_t<L64, double, float>;
    constexpr int CE = 16 / sizeof(V);                    // elements per 16-byte chunk
    constexpr int NCH = (kSvTX + 2 + CE - 1) / CE;        // chunks per staged row
    constexpr int NST = NCH * (kSvTY + 2);                // chunks per staged plane
    constexpr int KL = (NST + kSvUnit - 1) / kSvUnit;     // chunks per thread
    __shared__ __align__(16) V ring[Q * PM];
    const int count = (int)hdr->count;
    const long long total = hdr->total;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ring0 = smem_u32(ring);
    for (long long u = blockIdx.x; u < total; u += gridDim.x) {
        const SvItem* itp = items + sv_find(unit0, count, u);
        const int unit = (int)(u - itp->unit0);
        const RelaxCoef<LT> k = sv_k<LT>(*itp);
        const int n = k.n;
        const int zd = itp->zd;
        LT* const in_l = static_cast<LT*>(itp->in);
        LT* const out_l = static_cast<LT*>(itp->out);
        const LT* const rhs = static_cast<const LT*>(itp->rhs);
        double* const u64 = itp->u64;
        const double* const f64 = itp->f64;
        const int sxd = itp->sxd;
        const LT alpha = sv_alpha<LT>(*itp);
        const double alpha64 = itp->alpha64, beta64 = itp->beta64;
        const double n1 = itp->nscale, n0 = -6.0 * n1;   // NORM: L(., 1/h^2) (centre, the six others)
        Coefs<V> cf;
        if constexpr (OP == SV_K1 || L64) cf = itp->c64;
        else cf = itp->c;
        (void)n0;
        int XT, YT, ZT;
        sv_ring_units(n, zd, XT, YT, ZT);
        const int x0 = (unit % XT) * kSvTX, y0 = ((unit / XT) % YT) * kSvTY, z0 = (unit / (XT * YT)) * zd;
        const int z1 = min(z0 + zd, n);
        const V* src;
        int sx;
        if constexpr (OP == SV_K1) {
            src = reinterpret_cast<const V*>(u64);
            sx = sxd;
        } else {
            src = in_l;
            sx = k.sx;
        }
        const long long Sz = (long long)sx * (n + 2);
        // this thread's staging chunks: row r (y = y0 - 1 + r), chunk c (grown x = x0 + c*CE)
        const V* sp[KL];
        uint32_t sdst[KL];
        bool stg[KL];
#pragma unroll
        for (int q = 0; q < KL; q++) {
            const int t = threadIdx.x + q * kSvUnit;
            const int sr = t / NCH, sc_ = t % NCH;
            const int gx = x0 + sc_ * CE, gy = y0 - 1 + sr;
            stg[q] = t < NST && gx < min(x0 + kSvTX + 2, n + 2) && gy <= n;
            sp[q] = src + (stg[q] ? (long long)gx + (long long)sx * (gy + 1) + Sz * (z0 + 1) : 0);
            sdst[q] = ring0 + (uint32_t)sizeof(V) * (sr * RS + sc_ * CE);
        }
        auto stage = [&](int zz, int slot) {
            if (zz < z1) {
#pragma unroll
                for (int q = 0; q < KL; q++)
                    if (stg[q]) {
                        cp_async16(sdst[q] + (uint32_t)sizeof(V) * slot * PM, sp[q]);
                        sp[q] += Sz;
                    }
            }
            cp_async_commit();
        };
#pragma unroll
        for (int q = 0; q < L; q++) stage(z0 + q, q);
        constexpr int YC = kSvYC;
        const int x = x0 + lane, ya = y0 + YC * warp;      // this thread's cells: (x, ya + r), r < YC
        const bool xin = x < n;
        const V* col = src + (long long)grown_index<V>(n, sx, xin ? x : 0, ya < n ? ya : 0, z0);   // (x, ya, z0)
        bool act[YC];
        int ey[YC];
        V zm[YC], zc[YC];
#pragma unroll
        for (int r = 0; r < YC; r++) {
            act[r] = xin && ya + r < n;
            ey[r] = act[r] ? edge_code(ya + r, n) : 0;
            zm[r] = act[r] ? col[r * sx - Sz] : V(0);
            zc[r] = act[r] ? col[r * sx] : V(0);
        }
        const int ex = xin ? edge_code(x, n) : 0;
        const int cidx = (YC * warp + 1) * RS + lane + 1;  // cell (x, ya) in a ring plane
        int i = act[0] ? x + n * (ya + n * z0) : 0;        // (x, ya, z) in the n^3 fields
        // the grown field this phase writes (RELAX / NORM: out, K1: in, UPDATE: u64): cell (x, ya, z0),
        // advanced one plane per z step, and the offsets of the periodic images of this thread's
        // cells (x and y per thread and row, z per plane; 0 where there is none)
        using Wt = std::conditional_t<OP == SV_UPDATE, double, LT>;
        Wt* const wbase = OP == SV_UPDATE ? reinterpret_cast<Wt*>(u64) : reinterpret_cast<Wt*>(OP == SV_K1 ? in_l : out_l);
        const int wsx = OP == SV_UPDATE ? sxd : k.sx;
        const long long wSz = (long long)wsx * (n + 2);
        Wt* wp = wbase + (act[0] ? grown_index<Wt>(n, wsx, x, ya, z0) : 0);
        const int oxo = ex == 1 ? n : (ex == 2 ? -n : 0);
        int oyo[YC];
#pragma unroll
        for (int r = 0; r < YC; r++) oyo[r] = ey[r] == 1 ? n * wsx : (ey[r] == 2 ? -n * wsx : 0);
        const long long ozn = (long long)n * wSz;
        double m = 0.0;
        bool bad = false;     // K1 / NORM: a residual that is not finite (the norm itself skips NaN, as
                              // Reduction<Abs> does); the solve's norm is then reported as +inf
        // v at q (a valid cell) and at its periodic images (the stores store_with_images makes)
        auto put = [&](Wt* q, int oy, long long oz, Wt v) {
            *q = v;
            if ((oxo | oy) == 0 && oz == 0) return;
            if (oxo) q[oxo] = v;
            if (oy) q[oy] = v;
            if (oxo && oy) q[oxo + oy] = v;
            if (oz) {
                q[oz] = v;
                if (oxo) q[oz + oxo] = v;
                if (oy) q[oz + oy] = v;
                if (oxo && oy) q[oz + oxo + oy] = v;
            }
        };
        // one cell: the stencil taps, the plane's pointwise inputs and the outputs of this phase
        auto cell = [&](Wt* q, int oy, long long oz, int ii, V zm, V zc, V zp, V xm, V xp, V ym, V yp, LT rr,
                        double dd) {
            // Laplacian insertion order: 0, +x, -x, +y, -y, +z, -z
            if constexpr (OP == SV_K1) {
                double res;
                float al = 0.f;
                if (!k.helm) {
                    res = dadd(0.0, dd);
                    res = dadd(res, dmul(cf.c[0], (double)zc));
                    res = dadd(res, dmul(cf.c[1], (double)xp));
                    res = dadd(res, dmul(cf.c[2], (double)xm));
                    res = dadd(res, dmul(cf.c[3], (double)yp));
                    res = dadd(res, dmul(cf.c[4], (double)ym));
                    res = dadd(res, dmul(cf.c[5], (double)zp));
                    res = dadd(res, dmul(cf.c[6], (double)zm));
                } else {
                    double lp = 0.0;
                    lp = dadd(lp, dmul(cf.c[0], (double)zc));
                    lp = dadd(lp, dmul(cf.c[1], (double)xp));
                    lp = dadd(lp, dmul(cf.c[2], (double)xm));
                    lp = dadd(lp, dmul(cf.c[3], (double)yp));
                    lp = dadd(lp, dmul(cf.c[4], (double)ym));
                    lp = dadd(lp, dmul(cf.c[5], (double)zp));
                    lp = dadd(lp, dmul(cf.c[6], (double)zm));
                    res = dsub(dd, dsub(dmul(alpha64, (double)zc), dmul(beta64, lp)));
                    al = __double2float_rn(alpha64);
                }
                m = upd_abs(m, res);
                bad = bad || !(fabs(res) <= DBL_MAX);
                const float r32 = __double2float_rn(res);
                out_l[ii] = r32;
                put(q, oy, oz, relax_value(k, 0.f, 0.f, r32, al));
            } else {
                LT acc = LT(0);
                acc = dmadd(acc, cf.c[0], (LT)zc);
                acc = dmadd(acc, cf.c[1], (LT)xp);
                acc = dmadd(acc, cf.c[2], (LT)xm);
                acc = dmadd(acc, cf.c[3], (LT)yp);
                acc = dmadd(acc, cf.c[4], (LT)ym);
                acc = dmadd(acc, cf.c[5], (LT)zp);
                acc = dmadd(acc, cf.c[6], (LT)zm);
                const LT v = relax_value(k, acc, (LT)zc, rr, alpha);
                if constexpr (OP == SV_NORM) {
                    // the FP64 solver's norm: Poisson (0 - rho) + L(phi, 1/h^2); Helmholtz
                    // rho - (alpha*phi - beta*L(phi, 1/h^2)), whose sum is the sweep's own
                    double r2;
                    if (!k.helm) {
                        r2 = dsub(0.0, (double)rr);
                        r2 = dadd(r2, dmul(n0, (double)zc));
                        r2 = dadd(r2, dmul(n1, (double)xp));
                        r2 = dadd(r2, dmul(n1, (double)xm));
                        r2 = dadd(r2, dmul(n1, (double)yp));
                        r2 = dadd(r2, dmul(n1, (double)ym));
                        r2 = dadd(r2, dmul(n1, (double)zp));
                        r2 = dadd(r2, dmul(n1, (double)zm));
                    } else {
                        r2 = dsub((double)rr, dsub(dmul((double)alpha, (double)zc), dmul((double)k.beta, (double)acc)));
                    }
                    m = upd_abs(m, r2);
                    bad = bad || !(fabs(r2) <= DBL_MAX);
                    put(q, oy, oz, v);
                } else if constexpr (OP == SV_RELAX) {
                    put(q, oy, oz, v);
                } else {
                    put(q, oy, oz, dadd(dd, (double)v));
                }
            }
        };
        if constexpr (PB == 2) {
            // PB planes per block barrier: the ring holds planes z .. z + L + PB - 1 while planes
            // z .. z + PB - 1 are computed (their z neighbours from registers and the ring)
            int qz = 0;
            for (int z = z0; z < z1; z += PB) {
                LT rr[PB][YC];
                double dd[PB][YC];
#pragma unroll
                for (int h = 0; h < PB; h++)
#pragma unroll
                    for (int r = 0; r < YC; r++) {
                        rr[h][r] = LT(0);
                        dd[h][r] = 0.0;
                        const bool ok = act[r] && z + h < z1;
                        const int ih = i + h * n * n + r * n;
                        if constexpr (OP == SV_K1) {
                            if (ok) dd[h][r] = f64[ih];
                        } else {
                            if (ok) rr[h][r] = rhs[ih];
                        }
                        if constexpr (OP == SV_UPDATE) {
                            if (ok) dd[h][r] = wp[h * wSz + r * wsx];
                        }
                    }
                cp_async_wait<L - 1 - PB>();   // this thread's copies of planes up to z + PB have landed
                __syncthreads();               // everyone's have; everyone is done with planes z - PB .. z - 1
#pragma unroll
                for (int h = 0; h < PB; h++) stage(z + L + h, qz - PB + h >= 0 ? qz - PB + h : qz - PB + h + Q);
#pragma unroll
                for (int h = 0; h < PB; h++) {
                    if (z + h >= z1) break;
                    const int zz = z + h;
                    const int qh = qz + h >= Q ? qz + h - Q : qz + h;
                    if (act[0]) {
                        int q1 = qh + 1;
                        if (q1 >= Q) q1 -= Q;
                        const V* pl = ring + qh * PM + cidx;
                        V zp[YC];
                        if (zz + 1 < z1) {
#pragma unroll
                            for (int r = 0; r < YC; r++) zp[r] = ring[q1 * PM + cidx + r * RS];
                        } else {
#pragma unroll
                            for (int r = 0; r < YC; r++) zp[r] = act[r] ? col[Sz + r * sx] : V(0);
                        }
                        const long long oz = zz == 0 ? ozn : (zz == n - 1 ? -ozn : 0);
#pragma unroll
                        for (int r = 0; r < YC; r++) {
                            if (!act[r]) break;
                            // y neighbours: this thread's rows from registers, the tile's edge rows from the ring
                            const V ym = r == 0 ? pl[-RS] : zc[r - 1];
                            const V yp = (r + 1 < YC && act[r + 1]) ? zc[r + 1] : pl[(r + 1) * RS];
                            cell(wp + r * wsx, oyo[r], oz, i + r * n, zm[r], zc[r], zp[r], pl[r * RS - 1], pl[r * RS + 1],
                                 ym, yp, rr[h][r], dd[h][r]);
                        }
#pragma unroll
                        for (int r = 0; r < YC; r++) {
                            zm[r] = zc[r];
                            zc[r] = zp[r];
                        }
                    }
                    col += Sz;
                    wp += wSz;
                    i += n * n;
                }
                qz = qz + PB >= Q ? qz + PB - Q : qz + PB;
            }
        } else {
            int qz = 0;
            for (int z = z0; z < z1; z++) {
                LT rr[YC];
                double dd[YC];
#pragma unroll
                for (int r = 0; r < YC; r++) {
                    rr[r] = LT(0);
                    dd[r] = 0.0;
                    if constexpr (OP == SV_K1) {
                        if (act[r]) dd[r] = f64[i + r * n];
                    } else {
                        if (act[r]) rr[r] = rhs[i + r * n];
                    }
                    if constexpr (OP == SV_UPDATE) {
                        if (act[r]) dd[r] = wp[r * wsx];
                    }
                }
                cp_async_wait<L - 2>();   // this thread's copies of plane z + 1 have landed (PB = 1)
                __syncthreads();          // everyone's have; everyone is done with plane z - 1
                stage(z + L, qz == 0 ? Q - 1 : qz - 1);
                if (act[0]) {
                    int q1 = qz + 1;
                    if (q1 >= Q) q1 -= Q;
                    const V* pl = ring + qz * PM + cidx;
                    V zp[YC];
                    if (z + 1 < z1) {
#pragma unroll
                        for (int r = 0; r < YC; r++) zp[r] = ring[q1 * PM + cidx + r * RS];
                    } else {
#pragma unroll
                        for (int r = 0; r < YC; r++) zp[r] = act[r] ? col[Sz + r * sx] : V(0);
                    }
                    const long long oz = z == 0 ? ozn : (z == n - 1 ? -ozn : 0);
#pragma unroll
                    for (int r = 0; r < YC; r++) {
                        if (!act[r]) break;
                        // y neighbours: this thread's rows from registers, the tile's edge rows from the ring
                        const V ym = r == 0 ? pl[-RS] : zc[r - 1];
                        const V yp = (r + 1 < YC && act[r + 1]) ? zc[r + 1] : pl[(r + 1) * RS];
                        cell(wp + r * wsx, oyo[r], oz, i + r * n, zm[r], zc[r], zp[r], pl[r * RS - 1], pl[r * RS + 1], ym,
                             yp, rr[r], dd[r]);
                    }
#pragma unroll
                    for (int r = 0; r < YC; r++) {
                        zm[r] = zc[r];
                        zc[r] = zp[r];
                    }
                }
                col += Sz;
                wp += wSz;
                i += n * n;
                qz = qz == Q - 1 ? 0 : qz + 1;
            }
        }
        cp_async_wait<0>();
        __syncthreads();              // the ring is free for the next unit
        if constexpr (OP == SV_K1 || OP == SV_NORM) {
            if (__any_sync(0xffffffffu, bad)) m = CUDART_INF;
            for (int o = 16; o > 0; o >>= 1) {
                const double w = __shfl_down_sync(0xffffffffu, m, o);
                m = (m < w) ? w : m;
            }
            if (lane == 0 && m > 0.0) atomic_max_nonneg(norms + itp->slot, m);
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
template <typename T>
__global__ void __launch_bounds__(256) k_sv_fill(T* p, long long n, T v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

} // namespace pb
