// Level data: a patch layout in one device slab, its ghost exchange, and batched stencil steps.
//
// Reference counterparts (paths within the reference project):
//   LevelBoxData::define / exchange ........ include/base/implem/Proto_LevelBoxDataImplem.H:63-106, 315-329
//   LevelExchangeCopier::buildMotionPlans .. include/base/implem/Proto_LevelBoxDataImplem.H:900-951
//   Copier::makeItSoLocal .................. include/base/implem/Proto_CopierImplem.H:172-181
// The reference launches one copy kernel per motion item (up to 26 per patch) after a barrier.
// Here the motion plan is built once on the host (any disjoint tiling, uneven patch sizes
// allowed, periodic images included) and one kernel launch executes every item of the level.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include <type_traits>

#include "pb_internal.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

struct MotionItem {
    long long dOff, sOff;      // slab offsets of the destination / source patch (component 0)
    long long dvol, svol;      // grown-box volumes (component stride)
    int dlo[3], dS[3];         // destination grown box: low corner, extents
    int slo[3], sS[3];         // source grown box
    int rlo[3], rn[3];         // region, destination coordinates
    int sh[3];                 // source point = destination point - sh
};

__global__ void __launch_bounds__(256) k_exchange(double* slab, const MotionItem* __restrict__ items, int ncomp)
{
    const MotionItem it = items[blockIdx.x];
    const long long total = (long long)it.rn[0] * it.rn[1] * it.rn[2];
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        int x = it.rlo[0] + (int)(i % it.rn[0]);
        long long q = i / it.rn[0];
        int y = it.rlo[1] + (int)(q % it.rn[1]);
        int z = it.rlo[2] + (int)(q / it.rn[1]);
        long long di = (x - it.dlo[0]) + (long long)it.dS[0] * ((y - it.dlo[1]) + (long long)it.dS[1] * (z - it.dlo[2]));
        int sx = x - it.sh[0], sy = y - it.sh[1], sz = z - it.sh[2];
        long long si = (sx - it.slo[0]) + (long long)it.sS[0] * ((sy - it.slo[1]) + (long long)it.sS[1] * (sz - it.slo[2]));
        for (int c = 0; c < ncomp; c++) slab[it.dOff + c * it.dvol + di] = slab[it.sOff + c * it.svol + si];
    }
}

// Cross-rank halo transfer of a sharded level: one item per region of one local patch (source cells
// to pack, or ghost cells to fill) and its place in a contiguous buffer; gridDim.y blocks per item
// (blockIdx.x), consecutive threads on consecutive cells of the region (x fastest), components as
// blocks of the region's volume.
struct HaloItem {
    long long poff, gvol;      // slab offset and grown-box volume of the patch
    int glo[3], gS[3];         // grown box: low corner, extents
    int rlo[3], rn[3];         // region (patch coordinates)
    long long boff;            // buffer offset of the region's first component
};

__global__ void __launch_bounds__(256) k_halo(double* slab, double* buf, const HaloItem* __restrict__ items, int ncomp,
                                              int unpack)
{
    const HaloItem it = items[blockIdx.x];
    const long long vol = (long long)it.rn[0] * it.rn[1] * it.rn[2];
    for (long long i = (long long)blockIdx.y * blockDim.x + threadIdx.x; i < vol; i += (long long)gridDim.y * blockDim.x) {
        const int x = it.rlo[0] + (int)(i % it.rn[0]);
        const long long q = i / it.rn[0];
        const int y = it.rlo[1] + (int)(q % it.rn[1]), z = it.rlo[2] + (int)(q / it.rn[1]);
        const long long si = it.poff + (x - it.glo[0]) + (long long)it.gS[0] * ((y - it.glo[1]) + (long long)it.gS[1] * (z - it.glo[2]));
        for (int c = 0; c < ncomp; c++) {
            if (unpack) slab[si + c * it.gvol] = buf[it.boff + c * vol + i];
            else buf[it.boff + c * vol + i] = slab[si + c * it.gvol];
        }
    }
}

// One tile = a (tx x ty) block of (x, y) columns of one patch's valid box, each column walked over
// zd planes by one thread. The tile shape is chosen per patch-size class (the x extent of the
// valid box) by pb_level_autotune; the default is 16 x 16 columns, 8 planes deep.
struct PatchTile {
    long long off;             // slab offset of the patch
    int gS[3];                 // grown box extents
    int gh[3];                 // ghost widths (valid cell (0,0,0) sits at grown (gh0, gh1, gh2))
    int vn[3];                 // valid box extents
    int x0, y0, z0;            // tile origin in valid coordinates
    int tx, zd;                // threads along x (ty = 256 / tx) and planes per thread
    int xv;                    // x cells per thread (the tile is xv*tx cells wide)
    // face neighbours along each axis (tensor-product periodic tilings; read directly instead of
    // ghost cells): slab offset, valid extent and grown extent along that axis, low / high side
    long long nb_off[3][2];
    int nb_n[3][2];
    int nb_S[3][2];
};

constexpr int kLevelThreads = 256;

// out = u + a*S(u) (euler) or S(u) on the tile's points. z neighbours come from a (2R+1)-deep
// register window per column; x/y neighbours from global memory (L1). Terms are summed in the
// stencil's insertion order, so results are bitwise the one-point-per-thread kernel's.
template <class S>
__global__ void __launch_bounds__(kLevelThreads) k_level_star(const double* __restrict__ u, double* out,
                                                              const PatchTile* __restrict__ tiles, Coefs<double> cf,
                                                              double a, int euler)
{
    constexpr int R = S::R, W = 2 * R + 1;
    const PatchTile t = tiles[blockIdx.x];
    const int lx = threadIdx.x % t.tx, ly = threadIdx.x / t.tx;
    const int x = t.x0 + lx, y = t.y0 + ly;
    if (x >= t.vn[0] || y >= t.vn[1]) return;
    const long long Sx = t.gS[0], Sxy = (long long)t.gS[0] * t.gS[1];
    const int z1 = min(t.z0 + t.zd, t.vn[2]);
    const double* col = u + t.off + (x + t.gh[0]) + Sx * (y + t.gh[1]) + Sxy * t.gh[2];   // (x, y, z = 0)
    double* ocol = out + t.off + (x + t.gh[0]) + Sx * (y + t.gh[1]) + Sxy * t.gh[2];
    double win[W];
#pragma unroll
    for (int k = 0; k < 2 * R; k++) win[k] = __ldg(col + Sxy * (t.z0 - R + k));
    for (int z = t.z0; z < z1; z++) {
        win[2 * R] = __ldg(col + Sxy * (z + R));
        const double* c = col + Sxy * z;
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
            const double v = (oz != 0 || (ox == 0 && oy == 0)) ? win[R + oz] : __ldg(c + ox + Sx * oy);
            acc = dadd(acc, dmul(cf.c[j], v));
        }
        ocol[Sxy * z] = euler ? dadd(win[R], dmul(a, acc)) : acc;
#pragma unroll
        for (int k = 0; k < 2 * R; k++) win[k] = win[k + 1];
    }
}

// The same step on a periodic tensor-product tiling without ghost cells: a tap that leaves the
// patch along one axis (a star stencil moves along one axis at a time) reads the face neighbour's
// valid cell, which is what the exchange would have copied there. Bitwise the exchange + stencil.
// Each thread resolves, once, a column pointer and a plane stride per x/y tap (its own patch or a
// face neighbour); z taps that leave the patch read the z neighbour's plane (uniform per CTA).
template <class S>
__global__ void __launch_bounds__(kLevelThreads) k_level_star_fused(const double* __restrict__ u, double* out,
                                                                    const PatchTile* __restrict__ tiles,
                                                                    Coefs<double> cf, double a, int euler)
{
    constexpr int R = S::R, W = 2 * R + 1;
    const PatchTile t = tiles[blockIdx.x];
    const int lx = threadIdx.x % t.tx, ly = threadIdx.x / t.tx;
    const int x = t.x0 + lx, y = t.y0 + ly;
    const int nx = t.vn[0], ny = t.vn[1], nz = t.vn[2];
    if (x >= nx || y >= ny) return;
    const int g0 = t.gh[0], g1 = t.gh[1], g2 = t.gh[2];
    const long long Sx = t.gS[0], Sy = t.gS[1], Sxy = Sx * Sy;
    // (x, y, z = 0) of this patch and of the z neighbours (same x/y extents)
    const long long cxy = (x + g0) + Sx * (y + g1) + Sxy * g2;
    const double* col = u + t.off + cxy;
    const double* colzl = u + t.nb_off[2][0] + cxy + Sxy * t.nb_n[2][0];   // z' < 0 -> z' + nz_low
    const double* colzh = u + t.nb_off[2][1] + cxy;                          // z' >= nz -> z' - nz
    double* ocol = out + t.off + cxy;
    // x/y taps: column pointer and plane stride, resolved once
    const double* tp[S::NT];
    long long ts[S::NT];
#pragma unroll
    for (int j = 0; j < S::NT; j++) {
        const int ox = S::off(j, 0), oy = S::off(j, 1);
        tp[j] = col + ox + Sx * oy;
        ts[j] = Sxy;
        if (ox != 0 && x + ox < 0) {
            const long long Sq = t.nb_S[0][0];
            tp[j] = u + t.nb_off[0][0] + (x + ox + t.nb_n[0][0] + g0) + Sq * ((y + g1) + Sy * g2);
            ts[j] = Sq * Sy;
        } else if (ox != 0 && x + ox >= nx) {
            const long long Sq = t.nb_S[0][1];
            tp[j] = u + t.nb_off[0][1] + (x + ox - nx + g0) + Sq * ((y + g1) + Sy * g2);
            ts[j] = Sq * Sy;
        } else if (oy != 0 && y + oy < 0) {
            const long long Sq = t.nb_S[1][0];
            tp[j] = u + t.nb_off[1][0] + (x + g0) + Sx * ((y + oy + t.nb_n[1][0] + g1) + Sq * g2);
            ts[j] = Sx * Sq;
        } else if (oy != 0 && y + oy >= ny) {
            const long long Sq = t.nb_S[1][1];
            tp[j] = u + t.nb_off[1][1] + (x + g0) + Sx * ((y + oy - ny + g1) + Sq * g2);
            ts[j] = Sx * Sq;
        }
    }
    auto zcol = [&](int zz) -> double {
        if (zz >= nz) return __ldg(colzh + Sxy * (zz - nz));
        return __ldg((zz < 0 ? colzl : col) + Sxy * zz);
    };
    const int z1 = min(t.z0 + t.zd, nz);
#pragma unroll
    for (int j = 0; j < S::NT; j++) tp[j] += ts[j] * t.z0;   // advanced one plane per step below
    double* op = ocol + Sxy * t.z0;
    double win[W];
#pragma unroll
    for (int k = 0; k < 2 * R; k++) win[k] = zcol(t.z0 - R + k);
    for (int z = t.z0; z < z1; z++) {
        win[2 * R] = zcol(z + R);
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
            const double v = (oz != 0 || (ox == 0 && oy == 0)) ? win[R + oz] : __ldg(tp[j]);
            acc = dadd(acc, dmul(cf.c[j], v));
        }
        *op = euler ? dadd(win[R], dmul(a, acc)) : acc;
        op += Sxy;
#pragma unroll
        for (int j = 0; j < S::NT; j++) tp[j] += ts[j];
#pragma unroll
        for (int k = 0; k < 2 * R; k++) win[k] = win[k + 1];
    }
}

// Shared-memory variant of the fused step. Per z plane the CTA stages its (tx+2R) x (ty+2R) tile of
// the plane (halo cells from the face neighbours; the corner cells, which a star stencil never
// reads, are skipped) with per-thread asynchronous copies (cp.async) into a ring of kLevelRing(R)
// planes, kLevelLead planes ahead of the one being computed; x/y taps come from the ring, z taps
// from a per-column register window that is filled from the ring's centre column (from global
// memory for the R planes past the tile's z chunk). One barrier per plane. Bitwise the other two
// paths (same values, same term order).
constexpr int kLevelPlaneMax = (64 + 4) * (4 + 4);   // (tx+2R)(ty+2R) <= 544 for every tile shape at R <= 2
constexpr int kLevelPrefetch = 3;                    // planes in flight beyond the newest one waited for
__host__ __device__ constexpr int level_lead(int R) { return R + kLevelPrefetch; }
__host__ __device__ constexpr int level_ring(int R) { return level_lead(R) + 1; }


template <class S>
__global__ void __launch_bounds__(kLevelThreads) k_level_star_tiled(const double* __restrict__ u, double* out,
                                                                    const PatchTile* __restrict__ tiles,
                                                                    Coefs<double> cf, double a, int euler)
{
    constexpr int R = S::R, W = 2 * R + 1, L = level_lead(R), Q = level_ring(R);
    static_assert(R <= 2, "plane buffer sized for R <= 2");
    __shared__ __align__(16) double ring[Q * kLevelPlaneMax];
    const PatchTile t = tiles[blockIdx.x];
    const int tx = t.tx, ty = kLevelThreads / t.tx;
    const int BX = tx + 2 * R, BY = ty + 2 * R;
    const int nx = t.vn[0], ny = t.vn[1], nz = t.vn[2];
    const int g0 = t.gh[0], g1 = t.gh[1], g2 = t.gh[2];
    const long long Sx = t.gS[0], Sy = t.gS[1], Sxy = Sx * Sy;
    const int lx = threadIdx.x % tx, ly = threadIdx.x / tx;
    const int x = t.x0 + lx, y = t.y0 + ly;
    const bool act = x < nx && y < ny;
    const int z1 = min(t.z0 + t.zd, nz);
    // this thread's staging assignments are fixed across planes: base pointer and plane stride each
    constexpr int kMaxLoads = (kLevelPlaneMax + kLevelThreads - 1) / kLevelThreads;
    const double* lp[kMaxLoads];
    long long ls[kMaxLoads];
    bool lv_[kMaxLoads];
#pragma unroll
    for (int k = 0; k < kMaxLoads; k++) {
        const int i = threadIdx.x + k * kLevelThreads;
        const int hx = i % BX, hy = i / BX;
        const int xx = t.x0 - R + hx, yy = t.y0 - R + hy;
        const bool xo = xx < 0 || xx >= nx, yo = yy < 0 || yy >= ny;
        lv_[k] = i < BX * BY && !(xo && yo) && xx < nx + R && yy < ny + R;   // corners never read
        lp[k] = u;
        ls[k] = 0;
        if (!lv_[k]) continue;
        const double* p;
        long long st = Sxy;
        if (xx < 0) {
            const long long Sq = t.nb_S[0][0];
            p = u + t.nb_off[0][0] + (xx + t.nb_n[0][0] + g0) + Sq * ((yy + g1) + Sy * g2);
            st = Sq * Sy;
        } else if (xx >= nx) {
            const long long Sq = t.nb_S[0][1];
            p = u + t.nb_off[0][1] + (xx - nx + g0) + Sq * ((yy + g1) + Sy * g2);
            st = Sq * Sy;
        } else if (yy < 0) {
            const long long Sq = t.nb_S[1][0];
            p = u + t.nb_off[1][0] + (xx + g0) + Sx * ((yy + t.nb_n[1][0] + g1) + Sq * g2);
            st = Sx * Sq;
        } else if (yy >= ny) {
            const long long Sq = t.nb_S[1][1];
            p = u + t.nb_off[1][1] + (xx + g0) + Sx * ((yy - ny + g1) + Sq * g2);
            st = Sx * Sq;
        } else {
            p = u + t.off + (xx + g0) + Sx * (yy + g1) + Sxy * g2;
        }
        lp[k] = p + st * t.z0;
        ls[k] = st;
    }
    const uint32_t ring0 = smem_u32(ring) + 8u * threadIdx.x;
    // stage plane zz (< z1) into ring slot q; every call commits one group (empty past z1)
    auto stage = [&](int zz, int q) {
        if (zz < z1) {
#pragma unroll
            for (int k = 0; k < kMaxLoads; k++)
                if (lv_[k]) {
                    cp_async8(ring0 + 8u * (q * kLevelPlaneMax + k * kLevelThreads), lp[k]);
                    lp[k] += ls[k];
                }
        }
        cp_async_commit();
    };
    // own column (z taps) with its z neighbours
    const long long cxy = (x + g0) + Sx * (y + g1) + Sxy * g2;
    const double* col = u + t.off + cxy;
    const double* colzl = u + t.nb_off[2][0] + cxy + Sxy * t.nb_n[2][0];
    const double* colzh = u + t.nb_off[2][1] + cxy;
    auto zcol = [&](int zz) -> double {
        if (zz >= nz) return __ldg(colzh + Sxy * (zz - nz));
        return __ldg((zz < 0 ? colzl : col) + Sxy * zz);
    };
#pragma unroll
    for (int k = 0; k < L; k++) stage(t.z0 + k, k);
    double win[W];
    if (act) {
#pragma unroll
        for (int k = 0; k < 2 * R; k++) win[k] = zcol(t.z0 - R + k);
    }
    double* op = out + t.off + cxy + Sxy * t.z0;
    const int sc = (ly + R) * BX + (lx + R);
    int qz = 0;                          // ring slot of plane z
    for (int z = t.z0; z < z1; z++) {
        cp_async_wait<L - R - 1>();      // this thread's copies of plane z + R have landed
        __syncthreads();                 // everyone's have; everyone is done with plane z - 1
        const int qn = qz == 0 ? Q - 1 : qz - 1;   // slot of plane z - 1 = slot of plane z + L
        stage(z + L, qn);
        const double* pl = ring + qz * kLevelPlaneMax;
        if (act) {
            int qr = qz + R;
            if (qr >= Q) qr -= Q;
            win[2 * R] = z + R < z1 ? ring[qr * kLevelPlaneMax + sc] : zcol(z + R);
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < S::NT; j++) {
                const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
                const double v = (oz != 0 || (ox == 0 && oy == 0)) ? win[R + oz] : pl[sc + oy * BX + ox];
                acc = dadd(acc, dmul(cf.c[j], v));
            }
            *op = euler ? dadd(win[R], dmul(a, acc)) : acc;
#pragma unroll
            for (int k = 0; k < 2 * R; k++) win[k] = win[k + 1];
        }
        op += Sxy;
        qz = qz == Q - 1 ? 0 : qz + 1;
    }
    cp_async_wait<0>();                  // no copy outlives the block
}

// Two adjacent x cells per thread, for halo width 2 on layouts where every patch's x extent, the x
// ghost width and the slab are even (pb_level checks this): every staged pair of cells and every
// output pair then sits on a 16-byte boundary, so the ring is filled with 16-byte cp.async copies
// and the x/y taps are read as double2. The tile is (2 tx) x ty cells. Same terms in the same order
// per cell, so bitwise the one-cell paths.
constexpr int kLevelPairPlaneMax = (64 + 4) * (8 + 4);   // (2tx+4)(ty+4) <= 816 for tx in {8, 16, 32}


template <class S>
__global__ void __launch_bounds__(kLevelThreads, 4) k_level_star_pair(const double* __restrict__ u, double* out,
                                                                   const PatchTile* __restrict__ tiles,
                                                                   Coefs<double> cf, double a, int euler)
{
    // ring of Q = 2R+1 planes, lead L = Q-1: the z loop is unrolled by Q so ring slots and the
    // register window's slots are compile-time constants at every step (no window moves)
    constexpr int R = S::R, W = 2 * R + 1, Q = W, L = Q - 1, PM = kLevelPairPlaneMax;
    static_assert(R == 2, "cell pairs line up with 16-byte boundaries for a halo of 2");
    __shared__ __align__(16) double ring[Q * PM];
    const PatchTile t = tiles[blockIdx.x];
    const int tx = t.tx, ty = kLevelThreads / t.tx;
    const int BX = 2 * tx + 2 * R, BY = ty + 2 * R, PX = BX / 2;
    const int nx = t.vn[0], ny = t.vn[1], nz = t.vn[2];
    const int g0 = t.gh[0], g1 = t.gh[1], g2 = t.gh[2];
    const long long Sx = t.gS[0], Sy = t.gS[1], Sxy = Sx * Sy;
    const int lx = threadIdx.x % tx, ly = threadIdx.x / tx;
    const int x = t.x0 + 2 * lx, y = t.y0 + ly;
    const bool act = x < nx && y < ny;
    const int z0 = t.z0, z1 = min(t.z0 + t.zd, nz);
    constexpr int kMaxLoads = (PM / 2 + kLevelThreads - 1) / kLevelThreads;
    const double* lp[kMaxLoads];
    long long ls[kMaxLoads];
    bool lv_[kMaxLoads];
#pragma unroll
    for (int k = 0; k < kMaxLoads; k++) {
        const int i = threadIdx.x + k * kLevelThreads;   // pair index in the staged tile
        const int hx = i % PX, hy = i / PX;
        const int xx = t.x0 - R + 2 * hx, yy = t.y0 - R + hy;
        const bool xo = xx < 0 || xx >= nx, yo = yy < 0 || yy >= ny;
        lv_[k] = i < PX * BY && !(xo && yo) && xx < nx + R && yy < ny + R;   // corners never read
        lp[k] = u;
        ls[k] = 0;
        if (!lv_[k]) continue;
        const double* p;
        long long st = Sxy;
        if (xx < 0) {
            const long long Sq = t.nb_S[0][0];
            p = u + t.nb_off[0][0] + (xx + t.nb_n[0][0] + g0) + Sq * ((yy + g1) + Sy * g2);
            st = Sq * Sy;
        } else if (xx >= nx) {
            const long long Sq = t.nb_S[0][1];
            p = u + t.nb_off[0][1] + (xx - nx + g0) + Sq * ((yy + g1) + Sy * g2);
            st = Sq * Sy;
        } else if (yy < 0) {
            const long long Sq = t.nb_S[1][0];
            p = u + t.nb_off[1][0] + (xx + g0) + Sx * ((yy + t.nb_n[1][0] + g1) + Sq * g2);
            st = Sx * Sq;
        } else if (yy >= ny) {
            const long long Sq = t.nb_S[1][1];
            p = u + t.nb_off[1][1] + (xx + g0) + Sx * ((yy - ny + g1) + Sq * g2);
            st = Sx * Sq;
        } else {
            p = u + t.off + (xx + g0) + Sx * (yy + g1) + Sxy * g2;
        }
        lp[k] = p + st * t.z0;
        ls[k] = st;
    }
    const uint32_t ring0 = smem_u32(ring) + 16u * threadIdx.x;
    auto stage = [&](int zz, int q) {
        if (zz < z1) {
#pragma unroll
            for (int k = 0; k < kMaxLoads; k++)
                if (lv_[k]) {
                    cp_async16(ring0 + 8u * (q * PM + 2 * k * kLevelThreads), lp[k]);
                    lp[k] += ls[k];
                }
        }
        cp_async_commit();
    };
    const long long cxy = (x + g0) + Sx * (y + g1) + Sxy * g2;
    const double* col = u + t.off + cxy;
    const double* colzl = u + t.nb_off[2][0] + cxy + Sxy * t.nb_n[2][0];
    const double* colzh = u + t.nb_off[2][1] + cxy;
    auto zcol = [&](int zz) -> double2 {
        const double* q = zz >= nz ? colzh + Sxy * (zz - nz) : (zz < 0 ? colzl : col) + Sxy * zz;
        return __ldg(reinterpret_cast<const double2*>(q));
    };
#pragma unroll
    for (int k = 0; k < L; k++) stage(z0 + k, k);
    // window slot of plane p: (p - z0 + R) mod W
    double w0[W], w1[W];
    if (act) {
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            const double2 v = zcol(z0 - R + k);
            w0[k] = v.x;
            w1[k] = v.y;
        }
    }
    double* op = out + t.off + cxy + Sxy * t.z0;
    const int sc = (ly + R) * BX + (2 * lx + R);   // even: pairs are 16-byte aligned in the ring
    // one plane; J = (z - z0) mod Q, so plane z sits in ring slot J and window slot J + R
    auto step = [&](auto Jc, int z) {
        constexpr int J = decltype(Jc)::value;
        cp_async_wait<L - R - 1>();   // this thread's copies of plane z + R have landed
        __syncthreads();              // everyone's have; everyone is done with plane z - 1
        stage(z + L, (J + L) % Q);    // into the slot of plane z - 1
        if (act) {
            constexpr int qr = (J + R) % Q, wn = (J + 2 * R) % W;
            const double2 cn =
                z + R < z1 ? *reinterpret_cast<const double2*>(ring + qr * PM + sc) : zcol(z + R);
            w0[wn] = cn.x;
            w1[wn] = cn.y;
            const double* pl = ring + J * PM + sc;
            const double2 xm = *reinterpret_cast<const double2*>(pl - 2);   // x-2, x-1
            const double2 xc = *reinterpret_cast<const double2*>(pl);       // x, x+1
            const double2 xp = *reinterpret_cast<const double2*>(pl + 2);   // x+2, x+3
            const double2 ym1 = *reinterpret_cast<const double2*>(pl - BX);
            const double2 yp1 = *reinterpret_cast<const double2*>(pl + BX);
            const double2 ym2 = *reinterpret_cast<const double2*>(pl - 2 * BX);
            const double2 yp2 = *reinterpret_cast<const double2*>(pl + 2 * BX);
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int j = 0; j < S::NT; j++) {
                const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
                double v0, v1;
                if (oz != 0 || (ox == 0 && oy == 0)) {
                    const int ws = (J + R + oz + W) % W;
                    v0 = w0[ws];
                    v1 = w1[ws];
                } else if (oy != 0) {
                    const double2 q = oy == 1 ? yp1 : oy == -1 ? ym1 : oy == 2 ? yp2 : ym2;
                    v0 = q.x;
                    v1 = q.y;
                } else {
                    v0 = ox == -2 ? xm.x : ox == -1 ? xm.y : ox == 1 ? xc.y : xp.x;
                    v1 = ox == -2 ? xm.y : ox == -1 ? xc.x : ox == 1 ? xp.x : xp.y;
                }
                a0 = dadd(a0, dmul(cf.c[j], v0));
                a1 = dadd(a1, dmul(cf.c[j], v1));
            }
            constexpr int wc = (J + R) % W;
            double2 r;
            r.x = euler ? dadd(w0[wc], dmul(a, a0)) : a0;
            r.y = euler ? dadd(w1[wc], dmul(a, a1)) : a1;
            *reinterpret_cast<double2*>(op) = r;
        }
        op += Sxy;
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using I3 = std::integral_constant<int, 3>;
    using I4 = std::integral_constant<int, 4>;
    static_assert(Q == 5, "the unrolled loop below has five steps");
    for (int z = z0; z < z1; z += Q) {
        step(I0{}, z);
        if (z + 1 >= z1) break;
        step(I1{}, z + 1);
        if (z + 2 >= z1) break;
        step(I2{}, z + 2);
        if (z + 3 >= z1) break;
        step(I3{}, z + 3);
        if (z + 4 >= z1) break;
        step(I4{}, z + 4);
    }
    cp_async_wait<0>();
}

} // namespace pb

struct pb_level {
    std::vector<pb::Box3> patches;
    int ghost[3];
    pb::Box3 domain;
    int periodic[3];
    int ncomp;
    std::vector<long long> offsets;
    long long slab_elems;
    std::vector<pb::MotionItem> items;
    pb::MotionItem* d_items = nullptr;
    std::vector<pb::PatchTile> tiles;          // one cell per thread
    pb::PatchTile* d_tiles = nullptr;
    std::vector<pb::PatchTile> tiles2;         // two x cells per thread (fused halo-2 steps, pair_ok)
    pb::PatchTile* d_tiles2 = nullptr;
    bool pair_ok = false;                      // tensor tiling, even x extents and x ghost
    int device = 0;
    std::map<int, std::pair<int, int>> tune;   // valid x extent -> (tx, zd), one cell per thread
    std::map<int, std::pair<int, int>> tune2;  // the same for two cells per thread
    // periodic tensor-product tiling: face neighbour of patch i along axis d, side s
    bool tensor = false;
    bool tiled = true;                         // fused steps use the shared-memory tile kernel
    std::vector<int> nbr;                      // [i*6 + d*2 + s]
    // captured multi-step graph and what it was captured for
    cudaGraphExec_t graph = nullptr;
    std::vector<double> graph_key;
};

using namespace pb;

static void build_items(pb_level* lv)
{
    const int np = (int)lv->patches.size();
    long long L[3];
    for (int d = 0; d < 3; d++) L[d] = bsize(lv->domain, d);
    for (int i = 0; i < np; i++) {
        const Box3& vi = lv->patches[i];
        Box3 gi;
        for (int d = 0; d < 3; d++) { gi.lo[d] = vi.lo[d] - lv->ghost[d]; gi.hi[d] = vi.hi[d] + lv->ghost[d]; }
        for (int j = 0; j < np; j++) {
            const Box3& vj = lv->patches[j];
            Box3 gj;
            for (int d = 0; d < 3; d++) { gj.lo[d] = vj.lo[d] - lv->ghost[d]; gj.hi[d] = vj.hi[d] + lv->ghost[d]; }
            for (int sz = -1; sz <= 1; sz++)
                for (int sy = -1; sy <= 1; sy++)
                    for (int sx = -1; sx <= 1; sx++) {
                        int s[3] = {sx, sy, sz};
                        bool okp = true;
                        for (int d = 0; d < 3; d++) okp &= (s[d] == 0 || lv->periodic[d]);
                        if (!okp) continue;
                        if (i == j && sx == 0 && sy == 0 && sz == 0) continue;
                        Box3 img;
                        int sh[3];
                        for (int d = 0; d < 3; d++) {
                            sh[d] = (int)(s[d] * L[d]);
                            img.lo[d] = vj.lo[d] + sh[d];
                            img.hi[d] = vj.hi[d] + sh[d];
                        }
                        Box3 r = intersect(img, gi);
                        if (bempty(r)) continue;
                        MotionItem m;
                        m.dOff = lv->offsets[i];
                        m.sOff = lv->offsets[j];
                        m.dvol = bvol(gi);
                        m.svol = bvol(gj);
                        for (int d = 0; d < 3; d++) {
                            m.dlo[d] = gi.lo[d];
                            m.dS[d] = (int)bsize(gi, d);
                            m.slo[d] = gj.lo[d];
                            m.sS[d] = (int)bsize(gj, d);
                            m.rlo[d] = r.lo[d];
                            m.rn[d] = (int)bsize(r, d);
                            m.sh[d] = sh[d];
                        }
                        lv->items.push_back(m);
                    }
        }
    }
}

static std::pair<int, int> tile_shape(const pb_level* lv, int nx, int xv = 1)
{
    const auto& m = xv == 2 ? lv->tune2 : lv->tune;
    auto it = m.find(nx);
    if (it != m.end()) return it->second;
    return xv == 2 ? std::make_pair(16, 16) : std::make_pair(16, 8);
}

// Recognises a periodic tensor-product tiling (every patch = X_i x Y_j x Z_k of per-axis interval
// lists that tile the domain) and records each patch's face neighbours; other layouts keep the
// exchange + ghost-cell path.
static void detect_tensor(pb_level* lv)
{
    lv->tensor = false;
    lv->nbr.clear();
    for (int d = 0; d < 3; d++)
        if (!lv->periodic[d]) return;
    const int np = (int)lv->patches.size();
    std::vector<std::pair<int, int>> iv[3];
    for (int d = 0; d < 3; d++) {
        for (const Box3& b : lv->patches) iv[d].push_back({b.lo[d], b.hi[d]});
        std::sort(iv[d].begin(), iv[d].end());
        iv[d].erase(std::unique(iv[d].begin(), iv[d].end()), iv[d].end());
        int next = lv->domain.lo[d];
        for (auto& r : iv[d]) {
            if (r.first != next || r.second - r.first + 1 < lv->ghost[d]) return;   // gap, overlap or too thin
            next = r.second + 1;
        }
        if (next != lv->domain.hi[d] + 1) return;
    }
    const long long P0 = (long long)iv[0].size(), P1 = (long long)iv[1].size(), P2 = (long long)iv[2].size();
    if (P0 * P1 * P2 != np) return;
    std::vector<int> at(np, -1);
    std::vector<int> idx(3 * np);
    for (int i = 0; i < np; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            const Box3& b = lv->patches[i];
            c[d] = (int)(std::lower_bound(iv[d].begin(), iv[d].end(), std::make_pair(b.lo[d], b.hi[d])) - iv[d].begin());
            if (c[d] >= (int)iv[d].size() || iv[d][c[d]] != std::make_pair(b.lo[d], b.hi[d])) return;
            idx[3 * i + d] = c[d];
        }
        const long long k = c[0] + P0 * (c[1] + P1 * c[2]);
        if (at[k] >= 0) return;
        at[k] = i;
    }
    const long long P[3] = {P0, P1, P2};
    lv->nbr.assign(6 * np, -1);
    for (int i = 0; i < np; i++)
        for (int d = 0; d < 3; d++)
            for (int sd = 0; sd < 2; sd++) {
                long long c[3] = {idx[3 * i], idx[3 * i + 1], idx[3 * i + 2]};
                c[d] = (c[d] + (sd ? 1 : P[d] - 1)) % P[d];
                lv->nbr[6 * i + 2 * d + sd] = at[c[0] + P0 * (c[1] + P1 * c[2])];
            }
    lv->tensor = true;
}

static void build_tiles(pb_level* lv, int xv = 1, int only_nx = -1)
{
    std::vector<PatchTile>& tiles = xv == 2 ? lv->tiles2 : lv->tiles;
    tiles.clear();
    const int np = (int)lv->patches.size();
    for (int i = 0; i < np; i++) {
        const Box3& v = lv->patches[i];
        PatchTile t;
        t.off = lv->offsets[i];
        for (int d = 0; d < 3; d++) {
            t.gh[d] = lv->ghost[d];
            t.gS[d] = (int)bsize(v, d) + 2 * lv->ghost[d];
            t.vn[d] = (int)bsize(v, d);
        }
        if (only_nx >= 0 && t.vn[0] != only_nx) continue;
        for (int d = 0; d < 3; d++)
            for (int sd = 0; sd < 2; sd++) {
                const int q = lv->tensor ? lv->nbr[6 * i + 2 * d + sd] : i;
                const Box3& vq = lv->patches[q];
                t.nb_off[d][sd] = lv->offsets[q];
                t.nb_n[d][sd] = (int)bsize(vq, d);
                t.nb_S[d][sd] = (int)bsize(vq, d) + 2 * lv->ghost[d];
            }
        const std::pair<int, int> sh = tile_shape(lv, t.vn[0], xv);
        t.tx = sh.first;
        t.zd = sh.second;
        t.xv = xv;
        const int ty = kLevelThreads / t.tx;
        for (int z0 = 0; z0 < t.vn[2]; z0 += t.zd)
            for (int y0 = 0; y0 < t.vn[1]; y0 += ty)
                for (int x0 = 0; x0 < t.vn[0]; x0 += xv * t.tx) {
                    t.x0 = x0;
                    t.y0 = y0;
                    t.z0 = z0;
                    tiles.push_back(t);
                }
    }
}

static int upload_tiles(pb_level* lv, int xv = 1)
{
    std::vector<PatchTile>& tiles = xv == 2 ? lv->tiles2 : lv->tiles;
    PatchTile*& d = xv == 2 ? lv->d_tiles2 : lv->d_tiles;
    cudaFree(d);
    d = nullptr;
    if (tiles.empty()) return PB_OK;
    if (cudaMalloc(&d, tiles.size() * sizeof(PatchTile)) != cudaSuccess ||
        cudaMemcpy(d, tiles.data(), tiles.size() * sizeof(PatchTile), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return PB_ERR_CUDA;
    }
    return PB_OK;
}

// The two-cells-per-thread kernel applies: fused step of a halo-2 stencil, 16-byte aligned slabs.
static bool use_pairs(const pb_level* lv, int shape, bool fused, const void* u, const void* out)
{
    return fused && lv->tiled && lv->pair_ok && shape == 2 && ((uintptr_t)u % 16) == 0 && ((uintptr_t)out % 16) == 0;
}

static void drop_graph(pb_level* lv)
{
    if (lv->graph) cudaGraphExecDestroy(lv->graph);
    lv->graph = nullptr;
    lv->graph_key.clear();
}

// stencil coefficients (scale folded in) and its shape; PB_OK or an error status
static int level_coefs(const pb_level* lv, const pb_stencil* s, double scale, Coefs<double>& cf, int& shape)
{
    int nterms = 0;
    pb_box span;
    shape = 0;
    pb_stencil_info(s, &nterms, &span, &shape);
    if (shape != 1 && shape != 2) return PB_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; d++)
        if (-span.lo[d] > lv->ghost[d] || span.hi[d] > lv->ghost[d]) return PB_ERR_GHOST;
    double c[13];
    stencil_coefs(s, c, 13);
    for (int j = 0; j < 13; j++) cf.c[j] = 0.0;
    for (int j = 0; j < nterms; j++) cf.c[j] = (scale != 1.0) ? c[j] * scale : c[j];
    return PB_OK;
}

// fused: read face neighbours instead of ghost cells (tensor-product periodic tilings only)
static int launch_level_star(const pb_level* lv, int shape, const double* u, double* out, const Coefs<double>& cf,
                             double a, int euler, cudaStream_t st, bool fused = false)
{
    if (fused && !lv->tensor) return PB_ERR_ARG;
    if (use_pairs(lv, shape, fused, u, out)) {
        const unsigned np = (unsigned)lv->tiles2.size();
        if (np) k_level_star_pair<ShapeLap13><<<np, kLevelThreads, 0, st>>>(u, out, lv->d_tiles2, cf, a, euler);
        PB_LAUNCH_CHECK();
        return PB_OK;
    }
    const unsigned nb = (unsigned)lv->tiles.size();
    if (nb == 0) return PB_OK;
    if (fused && lv->tiled) {
        if (shape == 1) k_level_star_tiled<ShapeLap7><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
        else k_level_star_tiled<ShapeLap13><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
    } else if (fused) {
        if (shape == 1) k_level_star_fused<ShapeLap7><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
        else k_level_star_fused<ShapeLap13><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
    } else {
        if (shape == 1) k_level_star<ShapeLap7><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
        else k_level_star<ShapeLap13><<<nb, kLevelThreads, 0, st>>>(u, out, lv->d_tiles, cf, a, euler);
    }
    PB_LAUNCH_CHECK();
    return PB_OK;
}

struct pb_halo_plan {
    int ncomp = 1;
    int n = 0;
    int chunks = 1;            // blocks per item: the largest region over 2048 cells, at most 64
    long long elems = 0;
    pb::HaloItem* d_items = nullptr;
};

static int halo_run(const pb_halo_plan* hp, double* slab, double* buf, int unpack, cudaStream_t st)
{
    if (!hp || !slab || (!buf && hp->n > 0)) return PB_ERR_ARG;
    if (hp->n == 0) return PB_OK;
    k_halo<<<dim3(hp->n, hp->chunks), 256, 0, st>>>(slab, buf, hp->d_items, hp->ncomp, unpack);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

extern "C" {

int pb_halo_plan_create(const pb_level* lv, const pb_halo_item* items, int n, pb_halo_plan** out)
{
    if (!lv || !out || n < 0 || (n > 0 && !items)) return PB_ERR_ARG;
    std::vector<HaloItem> h;
    long long elems = 0, maxvol = 0;
    for (int k = 0; k < n; k++) {
        const int p = items[k].patch;
        if (p < 0 || p >= (int)lv->patches.size() || items[k].offset < 0) return PB_ERR_ARG;
        Box3 g = lv->patches[p];
        for (int d = 0; d < 3; d++) {
            g.lo[d] -= lv->ghost[d];
            g.hi[d] += lv->ghost[d];
        }
        const Box3 r = to_box(items[k].region);
        if (bempty(r) || !contains_box(g, r)) return PB_ERR_BOX;
        HaloItem it{};
        it.poff = lv->offsets[p];
        it.gvol = bvol(g);
        for (int d = 0; d < 3; d++) {
            it.glo[d] = g.lo[d];
            it.gS[d] = (int)bsize(g, d);
            it.rlo[d] = r.lo[d];
            it.rn[d] = (int)bsize(r, d);
        }
        it.boff = items[k].offset;
        elems = std::max(elems, it.boff + bvol(r) * lv->ncomp);
        maxvol = std::max(maxvol, bvol(r));
        h.push_back(it);
    }
    pb_halo_plan* hp = new (std::nothrow) pb_halo_plan;
    if (!hp) return PB_ERR_NOMEM;
    hp->ncomp = lv->ncomp;
    hp->n = n;
    hp->elems = elems;
    hp->chunks = (int)std::min<long long>(64, std::max<long long>(1, (maxvol + 2047) / 2048));
    if (n > 0 && (cudaMalloc(&hp->d_items, sizeof(HaloItem) * n) != cudaSuccess ||
                  cudaMemcpy(hp->d_items, h.data(), sizeof(HaloItem) * n, cudaMemcpyHostToDevice) != cudaSuccess)) {
        cudaGetLastError();
        cudaFree(hp->d_items);
        delete hp;
        return PB_ERR_CUDA;
    }
    *out = hp;
    return PB_OK;
}

int pb_halo_plan_destroy(pb_halo_plan* hp)
{
    if (!hp) return PB_OK;
    cudaFree(hp->d_items);
    delete hp;
    return PB_OK;
}

long long pb_halo_plan_elems(const pb_halo_plan* hp) { return hp ? hp->elems : -1; }

int pb_halo_pack_f64(const pb_halo_plan* hp, const double* slab, double* buffer, void* stream)
{
    return halo_run(hp, const_cast<double*>(slab), buffer, 0, (cudaStream_t)stream);
}

int pb_halo_unpack_f64(const pb_halo_plan* hp, double* slab, const double* buffer, void* stream)
{
    return halo_run(hp, slab, const_cast<double*>(buffer), 1, (cudaStream_t)stream);
}

int pb_level_create(const pb_box* patches, int npatch, const int ghost[3], pb_box domain, const int periodic[3],
                    int ncomp, pb_level** out)
{
    if (!patches || npatch < 1 || !ghost || !out || ncomp < 1) return PB_ERR_ARG;
    pb_level* lv = new (std::nothrow) pb_level;
    if (!lv) return PB_ERR_NOMEM;
    lv->domain = to_box(domain);
    lv->ncomp = ncomp;
    for (int d = 0; d < 3; d++) {
        lv->ghost[d] = ghost[d];
        lv->periodic[d] = periodic ? (periodic[d] != 0) : 0;
        if (ghost[d] < 0 || (lv->periodic[d] && ghost[d] > bsize(lv->domain, d))) { delete lv; return PB_ERR_ARG; }
    }
    long long off = 0;
    for (int i = 0; i < npatch; i++) {
        Box3 b = to_box(patches[i]);
        if (bempty(b) || !contains_box(lv->domain, b)) { delete lv; return PB_ERR_BOX; }
        lv->patches.push_back(b);
        lv->offsets.push_back(off);
        long long gv = 1;
        for (int d = 0; d < 3; d++) gv *= bsize(b, d) + 2 * ghost[d];
        off += gv * ncomp;
        off = (off + 31) / 32 * 32;   // every patch starts 256-byte aligned
    }
    lv->slab_elems = off;
    build_items(lv);
    detect_tensor(lv);
    lv->pair_ok = lv->tensor && ncomp == 1 && ghost[0] % 2 == 0;
    for (const Box3& b : lv->patches) lv->pair_ok = lv->pair_ok && bsize(b, 0) % 2 == 0;
    build_tiles(lv);
    if (lv->pair_ok) build_tiles(lv, 2);
    cudaGetDevice(&lv->device);
    if (!lv->items.empty()) {
        if (cudaMalloc(&lv->d_items, lv->items.size() * sizeof(MotionItem)) != cudaSuccess ||
            cudaMemcpy(lv->d_items, lv->items.data(), lv->items.size() * sizeof(MotionItem), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            cudaFree(lv->d_items);
            delete lv;
            return PB_ERR_CUDA;
        }
    }
    if (upload_tiles(lv) != PB_OK || upload_tiles(lv, 2) != PB_OK) {
        cudaFree(lv->d_items);
        cudaFree(lv->d_tiles);
        delete lv;
        return PB_ERR_CUDA;
    }
    *out = lv;
    return PB_OK;
}

int pb_level_destroy(pb_level* lv)
{
    if (!lv) return PB_OK;
    drop_graph(lv);
    cudaFree(lv->d_items);
    cudaFree(lv->d_tiles);
    cudaFree(lv->d_tiles2);
    delete lv;
    return PB_OK;
}

int pb_level_layout(const pb_level* lv, long long* offsets, long long* slab_elems, int* nitems)
{
    if (!lv) return PB_ERR_ARG;
    if (offsets) std::memcpy(offsets, lv->offsets.data(), lv->offsets.size() * sizeof(long long));
    if (slab_elems) *slab_elems = lv->slab_elems;
    if (nitems) *nitems = (int)lv->items.size();
    return PB_OK;
}

int pb_level_exchange_f64(const pb_level* lv, double* slab, void* stream)
{
    if (!lv || !slab) return PB_ERR_ARG;
    if (lv->items.empty()) return PB_OK;
    k_exchange<<<(unsigned)lv->items.size(), 256, 0, (cudaStream_t)stream>>>(slab, lv->d_items, lv->ncomp);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_level_stencil_f64(const pb_level* lv, const pb_stencil* s, int epilogue, const double* u_slab, double* out_slab,
                         double scale, double a, void* stream)
{
    if (!lv || !s || !u_slab || !out_slab) return PB_ERR_ARG;
    if (epilogue != 0 && epilogue != PB_EPI_EULER) return PB_ERR_ARG;
    if (lv->ncomp != 1) return PB_ERR_UNSUPPORTED;
    Coefs<double> cf;
    int shape, e;
    if ((e = level_coefs(lv, s, scale, cf, shape)) != PB_OK) return e;
    return launch_level_star(lv, shape, u_slab, out_slab, cf, a, epilogue == PB_EPI_EULER, (cudaStream_t)stream);
}

// 'steps' steps of: exchange(u), out = u + a*S(u) (or S(u)), swap; the result ends in u_slab. The
// launches are captured into one CUDA graph on the first call and replayed while the arguments
// stay the same (the graph holds the slab pointers).
int pb_level_steps_f64(pb_level* lv, const pb_stencil* s, int epilogue, double* u_slab, double* tmp_slab, double scale,
                       double a, int steps, void* stream)
{
    if (!lv || !s || !u_slab || !tmp_slab || steps < 0 || u_slab == tmp_slab) return PB_ERR_ARG;
    if (epilogue != 0 && epilogue != PB_EPI_EULER) return PB_ERR_ARG;
    if (lv->ncomp != 1) return PB_ERR_UNSUPPORTED;
    if (steps == 0) return PB_OK;
    Coefs<double> cf;
    int shape, e;
    if ((e = level_coefs(lv, s, scale, cf, shape)) != PB_OK) return e;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<double> key = {(double)(uintptr_t)u_slab, (double)(uintptr_t)tmp_slab, scale, a, (double)epilogue,
                               (double)steps, (double)shape, (double)(uintptr_t)lv->d_tiles,
                               (double)(uintptr_t)lv->d_tiles2};
    for (int j = 0; j < 13; j++) key.push_back(cf.c[j]);
    if (!lv->graph || key != lv->graph_key) {
        drop_graph(lv);
        cudaStream_t cs;
        PB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g;
        cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) { cudaStreamDestroy(cs); set_cuda_error(ce); return PB_ERR_CUDA; }
        double* a_ = u_slab;
        double* b_ = tmp_slab;
        for (int k = 0; k < steps && e == PB_OK; k++) {
            if (!lv->tensor && !lv->items.empty()) {
                k_exchange<<<(unsigned)lv->items.size(), 256, 0, cs>>>(a_, lv->d_items, lv->ncomp);
                if (cudaGetLastError() != cudaSuccess) e = PB_ERR_CUDA;
            }
            if (e == PB_OK) e = launch_level_star(lv, shape, a_, b_, cf, a, epilogue == PB_EPI_EULER, cs, lv->tensor);
            std::swap(a_, b_);
        }
        if (e == PB_OK && (steps & 1))
            if (cudaMemcpyAsync(u_slab, tmp_slab, sizeof(double) * lv->slab_elems, cudaMemcpyDeviceToDevice, cs) != cudaSuccess)
                e = PB_ERR_CUDA;
        ce = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (e != PB_OK) {
            if (ce == cudaSuccess) cudaGraphDestroy(g);
            return e;
        }
        if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
        ce = cudaGraphInstantiate(&lv->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { lv->graph = nullptr; set_cuda_error(ce); return PB_ERR_CUDA; }
        lv->graph_key = key;
    }
    PB_CUDA(cudaGraphLaunch(lv->graph, st));
    return PB_OK;
}

// Picks the tile shape (columns along x, planes per thread) for each patch-size class (valid x
// extent) by timing the stencil over that class's patches alone; the level keeps the choice.
int pb_level_autotune_f64(pb_level* lv, const pb_stencil* s, const double* u_slab, double* out_slab, double scale,
                          void* stream)
{
    if (!lv || !s || !u_slab || !out_slab) return PB_ERR_ARG;
    if (lv->ncomp != 1) return PB_ERR_UNSUPPORTED;
    Coefs<double> cf;
    int shape, e;
    if ((e = level_coefs(lv, s, scale, cf, shape)) != PB_OK) return e;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<int> classes;
    for (const Box3& b : lv->patches) classes.push_back((int)bsize(b, 0));
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    // the kernel the steps use: two cells per thread (tx up to 32, 64 cells) or one (tx up to 64)
    const int xv = use_pairs(lv, shape, lv->tensor, u_slab, out_slab) ? 2 : 1;
    auto& tune = xv == 2 ? lv->tune2 : lv->tune;
    static const int cand_tx[] = {8, 16, 32, 64};
    static const int cand_zd[] = {4, 8, 16, 32};
    const int ntx = xv == 2 ? 3 : 4;
    cudaEvent_t e0, e1;
    PB_CUDA(cudaEventCreate(&e0));
    PB_CUDA(cudaEventCreate(&e1));
    for (int nx : classes) {
        float best = 1e30f;
        std::pair<int, int> pick = tile_shape(lv, nx, xv);
        for (int ti = 0; ti < ntx; ti++) {
            const int tx = cand_tx[ti];
            if (xv * tx > 2 * nx && ti != 0) continue;   // mostly idle columns
            for (int zd : cand_zd) {
                tune[nx] = {tx, zd};
                build_tiles(lv, xv, nx);
                if ((e = upload_tiles(lv, xv)) != PB_OK) break;
                for (int w = 0; w < 2; w++) launch_level_star(lv, shape, u_slab, out_slab, cf, 0.0, 0, st, lv->tensor);
                cudaEventRecord(e0, st);
                for (int r = 0; r < 5; r++) launch_level_star(lv, shape, u_slab, out_slab, cf, 0.0, 0, st, lv->tensor);
                cudaEventRecord(e1, st);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) {
                    best = ms;
                    pick = {tx, zd};
                }
            }
            if (e != PB_OK) break;
        }
        tune[nx] = pick;
        if (e != PB_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    build_tiles(lv, xv);
    const int e2 = upload_tiles(lv, xv);
    drop_graph(lv);
    return e != PB_OK ? e : e2;
}

// The tile shape of each patch-size class used by the fused halo-2 step (the two-cells-per-thread
// tiles where the layout allows them): up to cap entries of (x extent, tile width in cells, planes).
int pb_level_tiles(const pb_level* lv, int* triples, int cap, int* n)
{
    if (!lv || !n || (cap > 0 && !triples)) return PB_ERR_ARG;
    std::vector<int> classes;
    for (const Box3& b : lv->patches) classes.push_back((int)bsize(b, 0));
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    int k = 0;
    for (int nx : classes) {
        if (k < cap) {
            const int xv = lv->pair_ok && lv->tiled ? 2 : 1;
            const std::pair<int, int> sh = tile_shape(lv, nx, xv);
            triples[3 * k] = nx;
            triples[3 * k + 1] = xv * sh.first;
            triples[3 * k + 2] = sh.second;
        }
        k++;
    }
    *n = std::min(k, cap);
    return PB_OK;
}

} // extern "C"
