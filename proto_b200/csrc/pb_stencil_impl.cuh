// Internal declarations shared by the stencil and multigrid modules.
#pragma once
#include "pb_internal.cuh"
#include "pb_star.cuh"

namespace pb {

constexpr int kMaxTerms = 256;

template <typename T>
struct TableArgs {
    T c[kMaxTerms];
    long long off[kMaxTerms];
    int n, ncomp, init_zero;
    Box3 sb, db, ib;
    int sr[3], dr[3], ds[3];
};

// Launch-shape knobs for the star kernels (set by the autotuner; defaults are heuristic).
struct StarTune {
    enum Mode { AUTO = 0, TMA = 1, SIMPLE = 2 };
    int mode = AUTO;
    long long min_tma_points = 1 << 18;   // smaller boxes are launch/latency bound: simple kernel
    int zc = 0;                          // z chunk per CTA; 0 = heuristic
    int ty = 8;                          // CTA height (rows of 64 points): 4, 8 or 16
};
StarTune& default_star_tune();
int cached_sm_count();
int grid_for(long long total, int threads);
// copies up to cap coefficients of a stencil (insertion order); returns the term count
int stencil_coefs(const pb_stencil* s, double* c, int cap);

// ---- star launch (shared with the multigrid module) -------------------------------------------
// TMA z-streaming launch with a CTA of 64 x TY threads; zc = 0 picks about six CTAs per SM.
template <class S, typename T, int TY, class Epi>
int launch_star_tma(const T* src, StarGeom g, const Coefs<T>& cf, const Epi& epi, cudaStream_t st, int zc)
{
    constexpr int EV = 16 / (int)sizeof(T);
    constexpr int NST = 2 * S::R + 4;
    using SM = StarSmem<S, T, TY>;
    g.pad = (g.ox - S::R) % EV;
    CUtensorMap map;
    int e = encode_tmap_3d(&map, src, (int)sizeof(T), g.Sx, g.Sy, g.Sz, SM::BX, SM::BY, 1);
    if (e != PB_OK) return e;
    int tiles = ((g.nx + kStarTX - 1) / kStarTX) * ((g.ny + TY - 1) / TY);
    if (zc <= 0) {
        long long want = (long long)cached_sm_count() * (6 * 8 / TY);
        zc = (int)(((long long)g.nz * tiles + want - 1) / want);
        if (zc < 8) zc = 8;
        zc = (zc + 7) / 8 * 8;
    }
    if (zc > g.nz) zc = g.nz;
    g.zc = zc;
    dim3 grid((g.nx + kStarTX - 1) / kStarTX, (g.ny + TY - 1) / TY, (g.nz + zc - 1) / zc);
    dim3 block(kStarTX, TY);
    size_t smem = (size_t)NST * SM::PLANE + NST * sizeof(uint64_t);
    auto kern = k_star_tma<S, T, TY, NST, Epi>;
    static bool attr_set = false;
    if (!attr_set) {
        PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    kern<<<grid, block, smem, st>>>(map, g, cf, epi);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

template <class S, typename T, class Epi>
int launch_star(const T* src, const Box3& srcBox, const Box3& ib, const Coefs<T>& cf, const Epi& epi,
                cudaStream_t st, const StarTune& tune)
{
    StarGeom g;
    g.nx = (int)bsize(ib, 0);
    g.ny = (int)bsize(ib, 1);
    g.nz = (int)bsize(ib, 2);
    g.ox = ib.lo[0] - srcBox.lo[0];
    g.oy = ib.lo[1] - srcBox.lo[1];
    g.oz = ib.lo[2] - srcBox.lo[2];
    g.Sx = (int)bsize(srcBox, 0);
    g.Sy = (int)bsize(srcBox, 1);
    g.Sz = (int)bsize(srcBox, 2);
    g.zc = g.nz;
    g.pad = 0;
    long long total = (long long)g.nx * g.ny * g.nz;
    bool use_tma = tune.mode != StarTune::SIMPLE && total >= tune.min_tma_points && g.ox >= S::R && tma_available();
    if (tune.mode == StarTune::TMA) use_tma = use_tma || (g.ox >= S::R && tma_available());
    if (use_tma) {
        int ty = tune.ty;
        int e;
        if (ty == 4) e = launch_star_tma<S, T, 4>(src, g, cf, epi, st, tune.zc);
        else if (ty == 16) e = launch_star_tma<S, T, 16>(src, g, cf, epi, st, tune.zc);
        else e = launch_star_tma<S, T, 8>(src, g, cf, epi, st, tune.zc);
        if (e == PB_OK || tune.mode == StarTune::TMA) return e;
    }
    int threads = 256;
    k_star_simple<S, T, Epi><<<grid_for(total, threads), threads, 0, st>>>(src, g, cf, epi);
    PB_LAUNCH_CHECK();
    return PB_OK;
}


} // namespace pb
