// Internal declarations shared by the stencil and multigrid modules.
#pragma once
#include <cmath>
#include <cstring>
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
    long long min_tma_points = 1 << 19;   // smaller boxes (64^3 and below) are launch/latency bound:
                                          // the simple kernel finishes them sooner
    int zc = 0;                          // z chunk per CTA; 0 = occupancy-based heuristic
    int ty = 8;                          // CTA tile height
    int yb = 2;                          // rows per consumer thread
    int xv = 0;                          // adjacent x points per consumer thread; (ty, yb, xv) in
                                         // {(8,1,1), (8,2,1), (8,2,2), (4,2,2)}; 0 = the caller's
                                         // default with ty 8, yb 2
    int nst = 0;                         // ring depth; 0 = as deep as two CTAs per SM allow (<= 2R+4)
    int aux_smem = 1;                    // stage auxiliary fields through shared memory by TMA
};
StarTune& default_star_tune();
int cached_sm_count();
int grid_for(long long total, int threads);
// copies up to cap coefficients of a stencil (insertion order); returns the term count
int stencil_coefs(const pb_stencil* s, double* c, int cap);

inline AuxSpecs no_aux()
{
    AuxSpecs a{};
    a.n = 0;
    a.in_smem = 0;
    return a;
}
// An auxiliary field of element size es stored on box fb, read at the points of index box ib.
inline AuxSpec aux_spec(const void* base, const Box3& fb, const Box3& ib, int es)
{
    AuxSpec a{};
    a.base = base;
    a.esize = es;
    a.Sx = (int)bsize(fb, 0);
    a.Sy = (int)bsize(fb, 1);
    a.Sz = (int)bsize(fb, 2);
    a.ox = ib.lo[0] - fb.lo[0];
    a.oy = ib.lo[1] - fb.lo[1];
    a.oz = ib.lo[2] - fb.lo[2];
    return a;
}

// ---- star launch (shared with the multigrid module) -------------------------------------------
template <class S, typename T, int TY, int YB, int XV, class Epi>
int launch_star_tma(const T* src, StarGeom g, const Coefs<T>& cf, const Epi& epi, cudaStream_t st, int zc,
                    AuxSpecs aux, int nst)
{
    constexpr int R = S::R;
    constexpr int EV = 16 / (int)sizeof(T);
    constexpr int NTHR = kStarTX * (TY / YB) + 32;
    using SM = StarSmem<S, T, TY, XV>;
    using AT = AuxTile<TY, XV>;
    if (XV > 1 && g.nx % XV != 0) return PB_ERR_ARG;
    g.pad = (g.ox - R) % EV;
    CUtensorMap map, amap[kMaxAux];
    int e = encode_tmap_3d(&map, src, (int)sizeof(T), g.Sx, g.Sy, g.Sz, SM::BX, SM::BY, 1);
    if (e != PB_OK) return e;
    memset(amap, 0, sizeof(amap));
    int aux_bytes = 0;
    if (aux.in_smem) {
        // every auxiliary field must be TMA-addressable; otherwise read them all from global memory
        for (int k = 0; k < aux.n && aux.in_smem; k++) {
            const AuxSpec& a = aux.a[k];
            if (a.ox < 0 || (a.esize != 4 && a.esize != 8) ||
                encode_tmap_3d(&amap[k], a.base, a.esize, a.Sx, a.Sy, a.Sz, AT::width(a.esize), TY, 1) != PB_OK)
                aux.in_smem = 0;
            else aux_bytes += AT::bytes(a.esize);
        }
        if (!aux.in_smem) aux_bytes = 0;
    }
    const size_t stage = (size_t)SM::PLANE + aux_bytes;
    if (nst <= 0) {
        // deepest ring (up to 2R+4 planes; 2R+3 for two x points per thread, measured faster for
        // the 256^3 FP64 sweep) that still lets the CTAs the registers allow share an SM
        const int per_sm = star_min_blocks(TY, YB, XV);
        nst = XV > 1 ? 2 * R + 3 : 2 * R + 4;
        while (nst > 2 * R + 1 && (size_t)per_sm * (nst * stage + 16 * nst + 1024) > 227 * 1024) nst--;
    }
    if (nst < 2 * R + 1 || nst > 16) return PB_ERR_ARG;
    g.nst = nst;
    const size_t smem = (size_t)nst * stage + 2 * nst * sizeof(uint64_t);
    if (smem > 220 * 1024) return PB_ERR_ARG;
    auto kern = k_star_tma<S, T, TY, YB, XV, Epi>;
    static int occ = 0;
    static bool attr_set = false;
    if (!attr_set) {
        PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        attr_set = true;
    }
    static size_t occ_smem = 0;
    if (occ == 0 || occ_smem != smem) {
        PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NTHR, smem));
        if (occ < 1) occ = 1;
        occ_smem = smem;
    }
    const long long tiles = (long long)((g.nx + SM::TXW - 1) / SM::TXW) * ((g.ny + TY - 1) / TY);
    if (zc <= 0) {
        // Pick the z chunk that best balances whole waves against the 2R+1 planes of halo each
        // CTA streams beyond its own: efficiency = (waves / ceil(waves)) * zc / (zc + 2R + 2).
        const double slots = (double)cached_sm_count() * occ;
        double best = -1.0;
        zc = g.nz;
        for (int c = 4; c <= g.nz; c += (c < 64 ? 2 : 8)) {
            const long long blocks = tiles * ((g.nz + c - 1) / c);
            const double waves = blocks / slots;
            const double eff = (waves / std::ceil(waves)) * c / (double)(c + 2 * R + 2);
            if (eff > best + 1e-9) {
                best = eff;
                zc = c;
            }
        }
    }
    if (zc > g.nz) zc = g.nz;
    g.zc = zc;
    dim3 grid((g.nx + SM::TXW - 1) / SM::TXW, (g.ny + TY - 1) / TY, (g.nz + zc - 1) / zc);
    kern<<<grid, NTHR, smem, st>>>(map, amap[0], amap[1], amap[2], g, aux, cf, epi);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

template <class S, typename T, class Epi>
int launch_star(const T* src, const Box3& srcBox, const Box3& ib, const Coefs<T>& cf, const Epi& epi,
                cudaStream_t st, const StarTune& tune, AuxSpecs aux = no_aux(), int xv_default = 1)
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
    g.nst = 0;
    if (aux.n > Epi::kAux) return PB_ERR_ARG;
    // unused auxiliary slots point at something harmless (their addresses are formed, never read)
    for (int k = aux.n; k < kMaxAux; k++) {
        aux.a[k] = AuxSpec{};
        aux.a[k].base = src;
        aux.a[k].esize = (int)sizeof(T);
    }
    if (aux.n == 0) aux.in_smem = 0;
    else aux.in_smem = aux.in_smem && tune.aux_smem;
    const long long total = (long long)g.nx * g.ny * g.nz;
    bool use_tma = tune.mode != StarTune::SIMPLE && total >= tune.min_tma_points && g.ox >= S::R && tma_available();
    if (tune.mode == StarTune::TMA) use_tma = g.ox >= S::R && tma_available();
    if (use_tma) {
        int e;
        const int xv = tune.xv ? tune.xv : xv_default;
        const bool pairs = xv == 2 && g.nx % 2 == 0;         // two x points per thread need an even extent
        if (pairs && tune.ty == 4) e = launch_star_tma<S, T, 4, 2, 2>(src, g, cf, epi, st, tune.zc, aux, tune.nst);
        else if (pairs) e = launch_star_tma<S, T, 8, 2, 2>(src, g, cf, epi, st, tune.zc, aux, tune.nst);
        else if (tune.yb == 1) e = launch_star_tma<S, T, 8, 1, 1>(src, g, cf, epi, st, tune.zc, aux, tune.nst);
        else e = launch_star_tma<S, T, 8, 2, 1>(src, g, cf, epi, st, tune.zc, aux, tune.nst);
        if (e == PB_OK || tune.mode == StarTune::TMA) return e;
    }
    const int threads = 256;
    k_star_simple<S, T, Epi><<<grid_for(total, threads), threads, 0, st>>>(src, g, aux, cf, epi);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

} // namespace pb
