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
#include <cmath>
#include <cstring>
#include <functional>
#include <type_traits>
#include <vector>

#include "pb_internal.cuh"
#include "pb_mg_kernels.cuh"
#include "pb_relax2.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

PB_DEFINE_ERROR_READER(read_error_mg)

template <typename T>
struct MGLevel {
    int n;
    int sx;              // x pitch of the grown layout
    double h, hsqinv;
    size_t grown_elems() const { return (size_t)sx * (n + 2) * (n + 2); }
    T* phi[2] = {nullptr, nullptr};
    T* rhs = nullptr;
    T* alpha = nullptr;
    int cur = 0;
};

// Inverse of the coarsest-level operator (N = n0^3 <= 512 cells), by Gauss-Jordan elimination with
// partial pivoting on [A | I]. A = L(., 1/h^2) (Poisson form) or diag(alpha) - beta*L(., 1/h^2)
// (Helmholtz form), periodic; when A is singular (Poisson, or alpha == 0 everywhere) the constant
// (6/h^2)/N is added to every entry, which fixes the mean of the solution. Row by row, the terms
// enter A in the order alpha, then the 7-point terms 0, +x, -x, +y, -y, +z, -z.
static bool coarse_inverse(int n0, double h, int helm, double beta, const double* alpha, std::vector<double>& inv)
{
    static const int off[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    static const double cc[7] = {-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
    const int N = n0 * n0 * n0;
    const double hs = 1. / (h * h);
    std::vector<double> M((size_t)N * 2 * N, 0.0);
    const size_t W = 2 * (size_t)N;
    bool singular = !helm;
    if (helm) {
        singular = true;
        for (int i = 0; i < N; i++) singular = singular && alpha[i] == 0.0;
    }
    for (int z = 0; z < n0; z++)
        for (int y = 0; y < n0; y++)
            for (int x = 0; x < n0; x++) {
                const int i = x + n0 * (y + n0 * z);
                if (helm) M[i * W + i] += alpha[i];
                for (int j = 0; j < 7; j++) {
                    const int qx = (x + off[j][0] + n0) % n0, qy = (y + off[j][1] + n0) % n0, qz = (z + off[j][2] + n0) % n0;
                    const int k = qx + n0 * (qy + n0 * qz);
                    const double t = helm ? (-beta) * (cc[j] * hs) : (cc[j] * hs);
                    M[i * W + k] += t;
                }
            }
    if (singular) {
        const double reg = (6.0 * hs) / N;
        for (int i = 0; i < N; i++)
            for (int k = 0; k < N; k++) M[i * W + k] += reg;
    }
    for (int i = 0; i < N; i++) M[i * W + N + i] = 1.0;
    for (int c = 0; c < N; c++) {
        int p = c;
        double best = std::fabs(M[c * W + c]);
        for (int r = c + 1; r < N; r++)
            if (std::fabs(M[r * W + c]) > best) {
                best = std::fabs(M[r * W + c]);
                p = r;
            }
        if (best == 0.0) return false;
        if (p != c)
            for (size_t j = 0; j < W; j++) std::swap(M[p * W + j], M[c * W + j]);
        const double piv = M[c * W + c];
        for (size_t j = 0; j < W; j++) M[c * W + j] = M[c * W + j] / piv;
        for (int r = 0; r < N; r++) {
            if (r == c) continue;
            const double f = M[r * W + c];
            if (f != 0.0)
                for (size_t j = 0; j < W; j++) M[r * W + j] = M[r * W + j] - f * M[c * W + j];
        }
    }
    inv.assign((size_t)N * N, 0.0);
    for (int i = 0; i < N; i++)
        for (int k = 0; k < N; k++) inv[(size_t)i * N + k] = M[i * W + N + k];
    return true;
}

} // namespace pb

struct pb_mg {
    pb_mg_params p;
    std::vector<pb::MGLevel<double>> lv;    // FP64 hierarchy, index 0 = coarsest (precision FP64)
    std::vector<pb::MGLevel<float>> lv32;   // FP32 hierarchy including the finest grid (precision MIXED)
    double* u64 = nullptr;                  // MIXED: FP64 solution, grown layout with periodic images
    double* f64 = nullptr;                  // MIXED: FP64 right-hand side, n^3
    double* alpha64 = nullptr;              // MIXED, Helmholtz: FP64 alpha, n^3
    double* ainv64 = nullptr;               // direct bottom solve: inverse of the coarsest operator
    float* ainv32 = nullptr;
    double* d_res = nullptr;
    double* h_res = nullptr;                // pinned
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_cur[2] = {0, 0};              // FP64: finest-level buffer index a graph leaves behind
    cudaStream_t graph_stream = nullptr;
    int device = 0;
};

using namespace pb;

static inline double lambda_of(const pb_mg_params& p, double h) { return (p.omega * (h * h)) / 6.0; }
static inline bool is_mixed(const pb_mg* mg) { return mg->p.precision == PB_MG_MIXED; }
static inline bool is_helm(const pb_mg* mg) { return mg->p.form == PB_MG_HELMHOLTZ; }

// the grown layout as a box: x spans the pitch (padding columns included), y and z one ghost layer
template <typename T>
static Box3 grown_box(const MGLevel<T>& L)
{
    Box3 b;
    for (int d = 0; d < 3; d++) { b.lo[d] = -1; b.hi[d] = L.n; }
    b.hi[0] = L.sx - 2;
    return b;
}
template <typename T>
static Box3 valid_box(const MGLevel<T>& L)
{
    Box3 b;
    for (int d = 0; d < 3; d++) { b.lo[d] = 0; b.hi[d] = L.n - 1; }
    return b;
}
template <typename T>
static RelaxCoef<T> relax_coef(const pb_mg* mg, const MGLevel<T>& L)
{
    RelaxCoef<T> k;
    k.n = L.n;
    k.sx = L.sx;
    k.helm = is_helm(mg);
    k.neg_lambda = (T)(-lambda_of(mg->p, L.h));
    k.beta = (T)mg->p.beta;
    k.omega = (T)mg->p.omega;
    k.diagB = (T)(6.0 * mg->p.beta * L.hsqinv);
    return k;
}
// rho (and alpha for the Helmholtz form) of a level as the star kernels' auxiliary fields
template <typename T>
static AuxSpecs level_aux(const pb_mg* mg, const T* rhs, const T* alpha, const MGLevel<T>& L)
{
    AuxSpecs a = no_aux();
    const Box3 vb = valid_box(L);
    a.n = is_helm(mg) ? 2 : 1;
    a.in_smem = 1;
    a.a[0] = aux_spec(rhs, vb, vb, (int)sizeof(T));
    if (is_helm(mg)) a.a[1] = aux_spec(alpha, vb, vb, (int)sizeof(T));
    return a;
}

template <typename T>
static int launch_relax(pb_mg* mg, MGLevel<T>& L, bool first, cudaStream_t st)
{
    const RelaxCoef<T> k = relax_coef(mg, L);
    if (first) {
        const long long total = (long long)L.n * L.n * L.n;
        k_relax_first<T><<<grid_for(total, 256), 256, 0, st>>>(L.rhs, L.alpha, L.phi[1 - L.cur], k);
        PB_LAUNCH_CHECK();
    } else {
        EpiRelax<T> epi;
        epi.out = L.phi[1 - L.cur];
        epi.k = k;
        const double s = is_helm(mg) ? L.hsqinv : mg->p.omega / 6.0;
        int e = launch_star<ShapeLap7>(L.phi[L.cur], grown_box(L), valid_box(L), lap7_coefs<T>(s), epi, st,
                                       default_star_tune(), level_aux(mg, L.rhs, L.alpha, L), 2);
        if (e != PB_OK) return e;
    }
    L.cur = 1 - L.cur;
    return PB_OK;
}

// ---- two sweeps per pass (k_relax2) ----------------------------------------------------------------
// Levels of edge >= g_relax2_min_edge whose edge the kernel is built for (128, 192, 256, 384) run each
// pair of consecutive sweeps as one k_relax2 pass; 0 turns this off (every sweep a launch). The
// results are bitwise the same either way.
static int g_relax2_min_edge = 128;
static int g_relax2_zc = 0;   // z chunk override (0: the occupancy heuristic)
static int g_relax2_pv = 0;   // cells per thread override (0: the default per edge)
static int g_relax2_rg = 0;   // output rows per group override (0: the default per edge)

// shared memory of a k_relax2 CTA with nst stages (the launcher's layout)
static size_t relax2_smem(int n, int esize, bool helm, int nst, int rg = 2, bool zero = false)
{
    int nb, bw;
    relax2_segments(esize == 8 ? grown_pitch<double>(n) : grown_pitch<float>(n), esize, &nb, &bw);
    const size_t tile0 = zero ? 0 : (size_t)(2 * rg + 4) * nb * bw, tilea = (size_t)(2 * rg + 2) * n;
    return nst * (tile0 + (helm ? 2 : 1) * tilea) * esize + 2 * tilea * esize + 16 * (size_t)nst;
}
// cells per thread: one at 128 and 256, two at 384 (a group of 192 threads is whole warps)
static int relax2_cells(int n)
{
    if (g_relax2_pv) return g_relax2_pv;
    return n == 384 ? 2 : 1;
}
// output rows per group: four (tiles of 8 rows) where three ring stages of them fit in the shared
// memory of the CTAs the kernel is built to keep resident per SM, else two (measured on B200: tiles
// of 8 rows where they fit take 6-16 % less time than tiles of 4)
static int relax2_rows(int n, int esize, bool helm)
{
    if (g_relax2_rg) return g_relax2_rg;
    const int per_sm = relax2_min_blocks(2 * (n / relax2_cells(n)) + 32);
    return (size_t)per_sm * (relax2_smem(n, esize, helm, 3, 4) + 1024) <= 227 * 1024 ? 4 : 2;
}
// the pass needs at least three stages (two planes in use and one in flight)
static bool relax2_edge(int n, int esize, bool helm)
{
    return g_relax2_min_edge > 0 && n >= g_relax2_min_edge && (n == 128 || n == 192 || n == 256 || n == 384) &&
           relax2_smem(n, esize, helm, 3, relax2_rows(n, esize, helm)) <= 220 * 1024 && tma_available();
}
template <typename T>
static bool relax2_ok(const pb_mg* mg, const MGLevel<T>& L)
{
    return relax2_edge(L.n, (int)sizeof(T), is_helm(mg));
}

template <typename T, int NXT, int PV, int RG, bool HELM, bool NORM, int MODE>
static int launch_relax2_t(pb_mg* mg, MGLevel<T>& L, double* result, cudaStream_t st)
{
    using SH = Relax2Shape<NXT, PV, RG>;
    constexpr bool ZERO = MODE == kRelax2Zero;
    Relax2Args<T> a;
    memset(&a, 0, sizeof(a));
    a.out = L.phi[1 - L.cur];
    if (MODE == kRelax2Update) {
        a.u = mg->u64;
        a.usx = grown_pitch<double>(L.n);
    }
    a.k = relax_coef(mg, L);
    a.c = lap7_coefs<T>(HELM ? L.hsqinv : mg->p.omega / 6.0);
    a.c2 = lap7_coefs<T>(L.hsqinv);
    a.beta = (T)mg->p.beta;
    a.result = result;
    relax2_segments(L.sx, (int)sizeof(T), &a.nb, &a.bw);
    // tile boxes (all rows of an x segment), and for the two tiles that wrap in y the boxes of all
    // rows but one plus single-row boxes
    CUtensorMap map, mapE, map1, rmap, rmapE, rmap1, amap, amapE, amap1;
    const int es = (int)sizeof(T), bwr = SH::N / (SH::N > 256 ? 2 : 1);
    int e = encode_tmap_3d(&map, L.phi[L.cur], es, L.sx, L.n + 2, L.n + 2, a.bw, SH::ROWS, 1);
    if (e == PB_OK) e = encode_tmap_3d(&mapE, L.phi[L.cur], es, L.sx, L.n + 2, L.n + 2, a.bw, SH::ROWS - 1, 1);
    if (e == PB_OK) e = encode_tmap_3d(&map1, L.phi[L.cur], es, L.sx, L.n + 2, L.n + 2, a.bw, 1, 1);
    if (e == PB_OK) e = encode_tmap_3d(&rmap, L.rhs, es, L.n, L.n, L.n, bwr, SH::B1ROWS, 1);
    if (e == PB_OK) e = encode_tmap_3d(&rmapE, L.rhs, es, L.n, L.n, L.n, bwr, SH::B1ROWS - 1, 1);
    if (e == PB_OK) e = encode_tmap_3d(&rmap1, L.rhs, es, L.n, L.n, L.n, bwr, 1, 1);
    if (e == PB_OK && HELM) e = encode_tmap_3d(&amap, L.alpha, es, L.n, L.n, L.n, bwr, SH::B1ROWS, 1);
    if (e == PB_OK && HELM) e = encode_tmap_3d(&amapE, L.alpha, es, L.n, L.n, L.n, bwr, SH::B1ROWS - 1, 1);
    if (e == PB_OK && HELM) e = encode_tmap_3d(&amap1, L.alpha, es, L.n, L.n, L.n, bwr, 1, 1);
    if (e != PB_OK) return e;
    if (!HELM) {
        amap = rmap;
        amapE = rmapE;
        amap1 = rmap1;
    }
    const int per_sm = relax2_min_blocks(SH::THREADS);
    int nst = 6;
    while (nst > 3 && (size_t)per_sm * (relax2_smem(SH::N, (int)sizeof(T), HELM, nst, RG, ZERO) + 1024) > 227 * 1024)
        nst--;
    a.nst = nst;
    const size_t smem = relax2_smem(SH::N, (int)sizeof(T), HELM, nst, RG, ZERO);
    if (smem > 220 * 1024) return PB_ERR_UNSUPPORTED;
    auto kern = k_relax2<T, NXT, PV, RG, HELM, NORM, MODE>;
    static bool attr = false;
    static int occ = 0;
    static size_t occ_smem = 0;
    if (!attr) {
        PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        attr = true;
    }
    if (occ_smem != smem) {
        PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, SH::THREADS, smem));
        if (occ < 1) occ = 1;
        occ_smem = smem;
    }
    // z chunk: whole waves of the resident CTAs against the 3 planes each chunk adds (2 of phi0 and
    // one of phi1 beyond its own)
    const int tiles = SH::N / SH::TY;
    const double slots = (double)cached_sm_count() * occ;
    double best = -1.0;
    int zc = SH::N;
    for (int c = 8; c <= SH::N; c += 2) {
        const long long blocks = (long long)tiles * ((SH::N + c - 1) / c);
        const double waves = blocks / slots;
        const double eff = (waves / std::ceil(waves)) * c / (double)(c + 3);
        if (eff > best + 1e-9) {
            best = eff;
            zc = c;
        }
    }
    // 384^3: chunks of 32 planes measured 1.5x faster than the wave heuristic's choice
    if (SH::N == 384) zc = 32;
    a.zc = g_relax2_zc > 0 ? std::min(g_relax2_zc, SH::N) : zc;
    dim3 grid(tiles, (SH::N + a.zc - 1) / a.zc);
    kern<<<grid, SH::THREADS, smem, st>>>(map, mapE, map1, rmap, rmapE, rmap1, amap, amapE, amap1, a);
    PB_LAUNCH_CHECK();
    if (MODE != kRelax2Update) L.cur = 1 - L.cur;
    return PB_OK;
}

template <typename T, bool HELM, bool NORM, int MODE>
static int launch_relax2_form(pb_mg* mg, MGLevel<T>& L, double* result, cudaStream_t st)
{
    // the pass that also takes the residual norm keeps tiles of 4 rows: its second tap sum makes
    // tiles of 8 rows spill (measured at 256^3: 132 us against 150 us)
    const bool tall = (g_relax2_rg || !NORM) && relax2_rows(L.n, (int)sizeof(T), HELM) == 4;
    const bool two = relax2_cells(L.n) == 2;
    switch (L.n) {
    case 128:
        if (two) return tall ? launch_relax2_t<T, 64, 2, 4, HELM, NORM, MODE>(mg, L, result, st)
                             : launch_relax2_t<T, 64, 2, 2, HELM, NORM, MODE>(mg, L, result, st);
        return tall ? launch_relax2_t<T, 128, 1, 4, HELM, NORM, MODE>(mg, L, result, st)
                    : launch_relax2_t<T, 128, 1, 2, HELM, NORM, MODE>(mg, L, result, st);
    case 256:
        if (two) return tall ? launch_relax2_t<T, 128, 2, 4, HELM, NORM, MODE>(mg, L, result, st)
                             : launch_relax2_t<T, 128, 2, 2, HELM, NORM, MODE>(mg, L, result, st);
        return tall ? launch_relax2_t<T, 256, 1, 4, HELM, NORM, MODE>(mg, L, result, st)
                    : launch_relax2_t<T, 256, 1, 2, HELM, NORM, MODE>(mg, L, result, st);
    case 192: return tall ? launch_relax2_t<T, 192, 1, 4, HELM, NORM, MODE>(mg, L, result, st)
                          : launch_relax2_t<T, 192, 1, 2, HELM, NORM, MODE>(mg, L, result, st);
    case 384: return tall ? launch_relax2_t<T, 192, 2, 4, HELM, NORM, MODE>(mg, L, result, st)
                          : launch_relax2_t<T, 192, 2, 2, HELM, NORM, MODE>(mg, L, result, st);
    default: return PB_ERR_UNSUPPORTED;
    }
}

// Two sweeps of level L in one pass (NORM: also the max-norm residual of the state it starts from,
// into result; MODE: from a zero state, or ending in the FP64 update). The caller checks relax2_ok.
template <typename T, bool NORM, int MODE = kRelax2Plain>
static int launch_relax2(pb_mg* mg, MGLevel<T>& L, double* result, cudaStream_t st)
{
    return is_helm(mg) ? launch_relax2_form<T, true, NORM, MODE>(mg, L, result, st)
                       : launch_relax2_form<T, false, NORM, MODE>(mg, L, result, st);
}

// last FP32 post-sweep of the finest level fused with u64 += e
static int launch_relax_update(pb_mg* mg, MGLevel<float>& L, cudaStream_t st)
{
    EpiRelaxUpdate epi;
    epi.u = mg->u64;
    epi.usx = grown_pitch<double>(L.n);
    epi.k = relax_coef(mg, L);
    const double s = is_helm(mg) ? L.hsqinv : mg->p.omega / 6.0;
    const AuxSpecs lvl = level_aux(mg, L.rhs, L.alpha, L);
    MGLevel<double> G;
    G.n = L.n;
    G.sx = epi.usx;
    AuxSpecs a = lvl;
    a.n = lvl.n + 1;
    a.a[0] = aux_spec(mg->u64, grown_box(G), valid_box(G), 8);
    a.a[1] = lvl.a[0];
    a.a[2] = lvl.a[1];
    return launch_star<ShapeLap7>(L.phi[L.cur], grown_box(L), valid_box(L), lap7_coefs<float>(s), epi, st,
                                  default_star_tune(), a, 2);
}

static int launch_resnorm(pb_mg* mg, MGLevel<double>& L, cudaStream_t st)
{
    PB_CUDA(cudaMemsetAsync(mg->d_res, 0, sizeof(double), st));
    EpiResnorm<double> epi;
    epi.helm = is_helm(mg);
    epi.beta = mg->p.beta;
    epi.result = mg->d_res;
    epi.m = 0.0;
    return launch_star<ShapeLap7>(L.phi[L.cur], grown_box(L), valid_box(L), lap7_coefs<double>(L.hsqinv), epi, st,
                                  default_star_tune(), level_aux(mg, L.rhs, L.alpha, L), 2);
}

// FP64, nu1 >= 1: the norm of the finest level's state fused with the next cycle's first sweep,
// which goes to the other buffer (L.cur is left on the state measured)
static bool fuse_norm(const pb_mg* mg) { return !is_mixed(mg) && mg->p.nu1 >= 1 && mg->p.levels >= 1; }

// sweeps the fused norm pass performs: two (k_relax2 with the norm) where that kernel takes the
// finest level and the cycle smooths at least twice before restricting, else one
static int norm_sweeps_for(const pb_mg_params& p)
{
    return (p.nu1 >= 2 && relax2_edge(p.n, 8, p.form == PB_MG_HELMHOLTZ)) ? 2 : 1;
}
static int norm_sweeps(const pb_mg* mg) { return norm_sweeps_for(mg->p); }

static int launch_relax_norm(pb_mg* mg, MGLevel<double>& L, cudaStream_t st)
{
    PB_CUDA(cudaMemsetAsync(mg->d_res, 0, sizeof(double), st));
    if (norm_sweeps(mg) == 2) {
        const int cur = L.cur;
        int e = launch_relax2<double, true>(mg, L, mg->d_res, st);
        L.cur = cur;   // left on the state measured, like the one-sweep pass
        return e;
    }
    EpiRelaxNorm<double> epi;
    epi.out = L.phi[1 - L.cur];
    epi.k = relax_coef(mg, L);
    epi.c2 = lap7_coefs<double>(L.hsqinv);
    epi.beta = mg->p.beta;
    epi.result = mg->d_res;
    epi.m = 0.0;
    const double s = is_helm(mg) ? L.hsqinv : mg->p.omega / 6.0;
    return launch_star<ShapeLap7>(L.phi[L.cur], grown_box(L), valid_box(L), lap7_coefs<double>(s), epi, st,
                                  default_star_tune(), level_aux(mg, L.rhs, L.alpha, L), 2);
}

// MIXED: FP64 residual of u64 + norm + FP32 right-hand side + first FP32 sweep of the finest level
// The mixed cycle runs its finest-level sweeps as two-sweep passes (the first pair from zero, the
// last ending in the FP64 update) where that kernel takes the level and both sweep counts are >= 2;
// otherwise the residual pass does the first sweep and a fused sweep the update.
static bool mixed_pairs(const pb_mg_params& p)
{
    return p.precision == PB_MG_MIXED && p.nu1 >= 2 && p.nu2 >= 2 &&
           relax2_edge(p.n, 4, p.form == PB_MG_HELMHOLTZ);
}

// FP64 residual of the solution: its max-norm into d_res, its FP32 copy as the finest FP32
// level's right-hand side, and (unless the cycle starts with a pair from zero) the first FP32 sweep.
static int launch_res64(pb_mg* mg, cudaStream_t st)
{
    MGLevel<float>& L = mg->lv32.back();
    PB_CUDA(cudaMemsetAsync(mg->d_res, 0, sizeof(double), st));
    EpiRes64 epi;
    epi.e32 = mixed_pairs(mg->p) ? nullptr : L.phi[1];
    epi.rhs32 = L.rhs;
    epi.helm = is_helm(mg);
    epi.beta = mg->p.beta;
    epi.k = relax_coef(mg, L);
    epi.result = mg->d_res;
    epi.m = 0.0;
    MGLevel<double> G;
    G.n = L.n;
    G.sx = grown_pitch<double>(L.n);
    G.h = L.h;
    G.hsqinv = L.hsqinv;
    const double s = is_helm(mg) ? L.hsqinv : -L.hsqinv;
    // one x point per consumer thread (measured at 384^3: 3 % faster solves than two; even at 256^3)
    int e = launch_star<ShapeLap7>((const double*)mg->u64, grown_box(G), valid_box(G), lap7_coefs<double>(s), epi, st,
                                   default_star_tune(), level_aux(mg, (const double*)mg->f64, (const double*)mg->alpha64, G), 1);
    L.cur = 1;
    return e;
}

template <typename T>
static int relax_sweeps(pb_mg* mg, MGLevel<T>& L, int k, bool zero_start, cudaStream_t st)
{
    int s = 0;
    if (zero_start && k >= 2 && relax2_ok(mg, L)) {
        // the first two sweeps from zero as one pass (no read of the zero state)
        int e = launch_relax2<T, false, kRelax2Zero>(mg, L, nullptr, st);
        if (e != PB_OK) return e;
        s = 2;
    } else if (zero_start && k > 0) {
        int e = launch_relax(mg, L, true, st);
        if (e != PB_OK) return e;
        s = 1;
    }
    if (relax2_ok(mg, L))
        for (; s + 2 <= k; s += 2) {
            int e = launch_relax2<T, false>(mg, L, nullptr, st);
            if (e != PB_OK) return e;
        }
    for (; s < k; s++) {
        int e = launch_relax(mg, L, false, st);
        if (e != PB_OK) return e;
    }
    if (zero_start && k == 0) PB_CUDA(cudaMemsetAsync(L.phi[L.cur], 0, sizeof(T) * L.grown_elems(), st));
    return PB_OK;
}

template <typename T>
static const T* bottom_inverse(const pb_mg* mg);
template <>
const double* bottom_inverse<double>(const pb_mg* mg) { return mg->ainv64; }
template <>
const float* bottom_inverse<float>(const pb_mg* mg) { return mg->ainv32; }

// Coarse levels at or below this edge run as one kernel (0: one launch per step everywhere). 8
// measured faster than 16 for a 256^3 solve: a 16^3 level runs sooner as separate launches.
static int g_coarse_edge = 8;

// Highest level index whose part of the cycle runs as one kernel, or -1.
static int fused_top(const pb_mg_params& p)
{
    if (g_coarse_edge <= 0) return -1;
    int ft = -1;
    for (int l = 0; l < p.levels && l < kMaxCoarse; l++)
        if ((p.n >> (p.levels - l)) <= g_coarse_edge) ft = l;
    return ft;
}

template <typename T>
static int launch_coarse_cycle(pb_mg* mg, std::vector<MGLevel<T>>& lv, int top, cudaStream_t st)
{
    CoarseArgs<T> a;
    memset(&a, 0, sizeof(a));
    const bool helm = is_helm(mg);
    for (int l = 0; l <= top; l++) {
        MGLevel<T>& L = lv[l];
        CoarseLevel<T>& c = a.lv[l];
        c.phi[0] = L.phi[0];
        c.phi[1] = L.phi[1];
        c.rhs = L.rhs;
        c.alpha = L.alpha;
        c.k = relax_coef(mg, L);
        c.crelax = lap7_coefs<T>(helm ? L.hsqinv : mg->p.omega / 6.0);
        c.cres = lap7_coefs<T>(helm ? L.hsqinv : -L.hsqinv);
    }
    a.top = top;
    a.nu1 = mg->p.nu1;
    a.nu2 = mg->p.nu2;
    a.nu_bottom = mg->p.nu_bottom;
    a.direct = mg->p.bottom == PB_MG_BOTTOM_DIRECT;
    a.ainv = bottom_inverse<T>(mg);
    a.beta = (T)mg->p.beta;
    CoarseOffsets off;
    memset(&off, 0, sizeof(off));
    const size_t smem = coarse_smem_layout(a, helm, off.o);
    static bool attr = false;
    if (!attr) {
        PB_CUDA(cudaFuncSetAttribute(k_coarse_cycle<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        attr = true;
    }
    a.in_smem = smem <= 216 * 1024 ? 1 : 0;   // the descriptor table takes a little static shared memory
    k_coarse_cycle<T><<<1, kCoarseThreads, a.in_smem ? smem : 0, st>>>(a, off);
    PB_LAUNCH_CHECK();
    for (int l = 0; l <= top; l++) lv[l].cur = 0;
    return PB_OK;
}

// Restriction of level L's residual into C's right-hand side: FP64 levels of edge >=
// g_restrict_star_edge through the TMA-staged star kernel (where it takes that path: 52 against
// 80 us at 256^3), else the z-marching kernel with x pairs from edge 64 (FP32 levels too: the
// staged kernel made 384^3 mixed solves 3 % slower, the paired kernel 3 % faster), the plain
// z-marching kernel below.
static int g_restrict_star_edge = 128;

template <typename T>
static int launch_restrict(pb_mg* mg, MGLevel<T>& L, MGLevel<T>& C, cudaStream_t st)
{
    const double s = is_helm(mg) ? L.hsqinv : -L.hsqinv;
    if (std::is_same<T, double>::value && g_restrict_star_edge > 0 && L.n >= g_restrict_star_edge && L.n % 2 == 0) {
        EpiRestrict<T> epi;
        epi.rhs_c = C.rhs;
        epi.nc = C.n;
        epi.helm = is_helm(mg);
        epi.beta = (T)mg->p.beta;
        epi.sum = T(0);
        StarTune tune = default_star_tune();
        tune.mode = StarTune::TMA;
        tune.ty = 8;
        tune.yb = 2;
        tune.xv = 2;
        tune.zc = 0;     // the chunk heuristic only picks even chunks; an even edge keeps every start even
        if (launch_star<ShapeLap7>(L.phi[L.cur], grown_box(L), valid_box(L), lap7_coefs<T>(s), epi, st, tune,
                                   level_aux(mg, L.rhs, L.alpha, L), 2) == PB_OK)
            return PB_OK;
        cudaGetLastError();
    }
    if (L.n >= 64 && L.n % 2 == 0) {   // x pairs: a warp covers 64 fine cells (3 % faster solves)
        const int c2 = restrict_x2_chunk(L.n, cached_sm_count());
        k_resid_restrict_x2<T><<<restrict_x2_grid(L.n, c2), dim3(32, 8), 0, st>>>(
            L.phi[L.cur], L.rhs, L.alpha, C.rhs, L.n, L.sx, is_helm(mg), lap7_coefs<T>(s), (T)mg->p.beta, c2);
        PB_LAUNCH_CHECK();
        return PB_OK;
    }
    const int czc = restrict_z_chunk(L.n, cached_sm_count());
    k_resid_restrict_z<T><<<restrict_z_grid(L.n, czc), dim3(32, 8), 0, st>>>(
        L.phi[L.cur], L.rhs, L.alpha, C.rhs, L.n, L.sx, is_helm(mg), lap7_coefs<T>(s), (T)mg->p.beta, czc);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

// V-cycle on level l of hierarchy lv. pre_done: the first pre-smoothing sweep(s) already ran (the
// mixed-precision residual pass does one, the FP64 norm pass one or two); fuse_update: the last
// post-smoothing sweep adds its result to the FP64 solution instead of storing it.
template <typename T>
static int vcycle(pb_mg* mg, std::vector<MGLevel<T>>& lv, int l, bool zero_start, int pre_done, bool fuse_update,
                  cudaStream_t st)
{
    MGLevel<T>& L = lv[l];
    if (zero_start) L.cur = 0;
    if (zero_start && l == fused_top(mg->p)) return launch_coarse_cycle(mg, lv, l, st);
    int e;
    if (l > 0) {
        MGLevel<T>& C = lv[l - 1];
        if ((e = relax_sweeps(mg, L, mg->p.nu1 - pre_done, zero_start && !pre_done, st)) != PB_OK) return e;
        if ((e = launch_restrict(mg, L, C, st)) != PB_OK) return e;
        if ((e = vcycle(mg, lv, l - 1, true, 0, false, st)) != PB_OK) return e;
        k_prolong<T><<<prolong_grid(L.n), dim3(32, 8), 0, st>>>(L.phi[L.cur], C.phi[C.cur], L.n, L.sx, C.sx);
        PB_LAUNCH_CHECK();
        if (!fuse_update) return relax_sweeps(mg, L, mg->p.nu2, false, st);
        if constexpr (std::is_same<T, float>::value) {
            if (mixed_pairs(mg->p)) {
                if ((e = relax_sweeps(mg, L, mg->p.nu2 - 2, false, st)) != PB_OK) return e;
                return launch_relax2<float, false, kRelax2Update>(mg, L, nullptr, st);
            }
            if ((e = relax_sweeps(mg, L, mg->p.nu2 - 1, false, st)) != PB_OK) return e;
            return launch_relax_update(mg, L, st);
        }
        return PB_ERR_ARG;
    }
    if (mg->p.bottom == PB_MG_BOTTOM_DIRECT) {
        const int N = L.n * L.n * L.n;
        k_bottom_direct<T><<<(N + 255) / 256, 256, 0, st>>>(bottom_inverse<T>(mg), L.rhs, L.phi[0], L.n, L.sx);
        PB_LAUNCH_CHECK();
        L.cur = 0;
        return PB_OK;
    }
    return relax_sweeps(mg, L, mg->p.nu_bottom, zero_start, st);
}

template <typename T>
static void free_levels(std::vector<MGLevel<T>>& lv)
{
    for (auto& L : lv) {
        cudaFree(L.phi[0]);
        cudaFree(L.phi[1]);
        cudaFree(L.alpha);
        cudaFree(L.rhs);
    }
    lv.clear();
}

static int mg_free(pb_mg* mg)
{
    free_levels(mg->lv);
    free_levels(mg->lv32);
    for (int k = 0; k < 2; k++)
        if (mg->graph[k]) cudaGraphExecDestroy(mg->graph[k]);
    if (mg->graph_stream) cudaStreamDestroy(mg->graph_stream);
    cudaFree(mg->u64);
    cudaFree(mg->f64);
    cudaFree(mg->alpha64);
    cudaFree(mg->ainv64);
    cudaFree(mg->ainv32);
    cudaFree(mg->d_res);
    cudaFreeHost(mg->h_res);
    delete mg;
    return PB_OK;
}

// One V-cycle on the finest level followed by the residual norm into h_res.
static int cycle_and_norm(pb_mg* mg, cudaStream_t st)
{
    int e;
    if (is_mixed(mg)) {
        const int top = (int)mg->lv32.size() - 1;
        if (mixed_pairs(mg->p)) {
            // the correction starts from zero: its first two sweeps are one pass
            if ((e = vcycle(mg, mg->lv32, top, true, 0, true, st)) != PB_OK) return e;
        } else {
            mg->lv32[top].cur = 1;   // the residual pass left the first sweep in phi[1]
            if ((e = vcycle(mg, mg->lv32, top, false, 1, true, st)) != PB_OK) return e;
        }
        if ((e = launch_res64(mg, st)) != PB_OK) return e;
    } else if (fuse_norm(mg)) {
        const int top = (int)mg->lv.size() - 1;
        MGLevel<double>& T = mg->lv[top];
        T.cur = 1 - T.cur;   // the previous fused pass left this cycle's first sweeps in the other buffer
        if ((e = vcycle(mg, mg->lv, top, false, norm_sweeps(mg), false, st)) != PB_OK) return e;
        if ((e = launch_relax_norm(mg, T, st)) != PB_OK) return e;
    } else {
        const int top = (int)mg->lv.size() - 1;
        if ((e = vcycle(mg, mg->lv, top, false, 0, false, st)) != PB_OK) return e;
        if ((e = launch_resnorm(mg, mg->lv[top], st)) != PB_OK) return e;
    }
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
    if (p->bottom != PB_MG_BOTTOM_RELAX && p->bottom != PB_MG_BOTTOM_DIRECT) return PB_ERR_ARG;
    const long long n0 = p->n >> p->levels;
    if (p->bottom == PB_MG_BOTTOM_DIRECT && n0 * n0 * n0 > 512) return PB_ERR_ARG;
    // the mixed cycle fuses its first pre-sweep and its last post-sweep of the finest grid
    if (p->precision == PB_MG_MIXED && (p->nu1 < 1 || p->nu2 < 1 || p->levels < 1)) return PB_ERR_ARG;
    return PB_OK;
}

template <typename T>
static bool alloc_levels(const pb_mg_params* p, std::vector<MGLevel<T>>& lv)
{
    lv.resize(p->levels + 1);
    for (int l = 0; l <= p->levels; l++) {
        MGLevel<T>& L = lv[l];
        L.n = p->n >> (p->levels - l);
        L.sx = grown_pitch<T>(L.n);
        L.h = (double)(1 << (p->levels - l)) / (double)p->n;
        L.hsqinv = 1. / (L.h * L.h);
        const size_t g = sizeof(T) * L.grown_elems();
        const size_t c = sizeof(T) * (size_t)L.n * L.n * L.n;
        bool ok = cudaMalloc(&L.phi[0], g) == cudaSuccess && cudaMalloc(&L.phi[1], g) == cudaSuccess &&
                  cudaMalloc(&L.rhs, c) == cudaSuccess;
        if (ok && p->form == PB_MG_HELMHOLTZ) ok = cudaMalloc(&L.alpha, c) == cudaSuccess;
        if (ok) ok = cudaMemset(L.phi[0], 0, g) == cudaSuccess && cudaMemset(L.phi[1], 0, g) == cudaSuccess;
        if (!ok) return false;
    }
    return true;
}

// Builds the coarsest-level inverse from the coarsest alpha held on the device (Helmholtz form)
// and uploads it in the solver's precision(s).
static int setup_bottom(pb_mg* mg)
{
    if (mg->p.bottom != PB_MG_BOTTOM_DIRECT) return PB_OK;
    const bool mixed = is_mixed(mg);
    const int n0 = mixed ? mg->lv32[0].n : mg->lv[0].n;
    const double h = mixed ? mg->lv32[0].h : mg->lv[0].h;
    const int N = n0 * n0 * n0;
    std::vector<double> alpha(N, 0.0);
    if (is_helm(mg)) {
        PB_CUDA(cudaDeviceSynchronize());
        if (mixed) {
            std::vector<float> a32(N);
            PB_CUDA(cudaMemcpy(a32.data(), mg->lv32[0].alpha, sizeof(float) * N, cudaMemcpyDeviceToHost));
            for (int i = 0; i < N; i++) alpha[i] = a32[i];
        } else {
            PB_CUDA(cudaMemcpy(alpha.data(), mg->lv[0].alpha, sizeof(double) * N, cudaMemcpyDeviceToHost));
        }
    }
    std::vector<double> inv;
    if (!coarse_inverse(n0, h, is_helm(mg), mg->p.beta, alpha.data(), inv)) return PB_ERR_ARG;
    if (mixed) {
        std::vector<float> inv32(inv.size());
        for (size_t i = 0; i < inv.size(); i++) inv32[i] = (float)inv[i];
        PB_CUDA(cudaMemcpy(mg->ainv32, inv32.data(), sizeof(float) * inv32.size(), cudaMemcpyHostToDevice));
    } else {
        PB_CUDA(cudaMemcpy(mg->ainv64, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice));
    }
    return PB_OK;
}

extern "C" {

long long pb_mg_device_bytes(const pb_mg_params* p)
{
    if (params_ok(p) != PB_OK) return -1;
    const bool mixed = p->precision == PB_MG_MIXED;
    const long long es = mixed ? 4 : 8;
    long long total = 0;
    for (int l = 0; l <= p->levels; l++) {
        const int n = p->n >> (p->levels - l);
        const long long g = (long long)(mixed ? grown_pitch<float>(n) : grown_pitch<double>(n)) * (n + 2) * (n + 2);
        total += 2 * g * es + (long long)n * n * n * es;
        if (p->form == PB_MG_HELMHOLTZ) total += (long long)n * n * n * es;
    }
    if (mixed) {
        const long long n = p->n;
        total += (long long)grown_pitch<double>(p->n) * (n + 2) * (n + 2) * 8 + n * n * n * 8;
        if (p->form == PB_MG_HELMHOLTZ) total += n * n * n * 8;
    }
    if (p->bottom == PB_MG_BOTTOM_DIRECT) {
        const long long n0 = p->n >> p->levels, N = n0 * n0 * n0;
        total += N * N * es;
    }
    return total + 256;
}

int pb_mg_create(const pb_mg_params* p, pb_mg** out)
{
    int e = params_ok(p);
    if (e != PB_OK) return e;
    if (!out) return PB_ERR_ARG;
    pb_mg* mg = new (std::nothrow) pb_mg;
    if (!mg) return PB_ERR_NOMEM;
    mg->p = *p;
    cudaGetDevice(&mg->device);
    bool ok;
    const long long n0 = p->n >> p->levels, N0 = n0 * n0 * n0;
    if (p->precision == PB_MG_MIXED) {
        const size_t n = (size_t)p->n, ug = 8 * (size_t)grown_pitch<double>(p->n) * (n + 2) * (n + 2);
        ok = alloc_levels(p, mg->lv32) && cudaMalloc(&mg->u64, ug) == cudaSuccess &&
             cudaMalloc(&mg->f64, 8 * n * n * n) == cudaSuccess && cudaMemset(mg->u64, 0, ug) == cudaSuccess;
        if (ok && p->form == PB_MG_HELMHOLTZ) ok = cudaMalloc(&mg->alpha64, 8 * n * n * n) == cudaSuccess;
        if (ok && p->bottom == PB_MG_BOTTOM_DIRECT) ok = cudaMalloc(&mg->ainv32, sizeof(float) * N0 * N0) == cudaSuccess;
    } else {
        ok = alloc_levels(p, mg->lv);
        if (ok && p->bottom == PB_MG_BOTTOM_DIRECT) ok = cudaMalloc(&mg->ainv64, sizeof(double) * N0 * N0) == cudaSuccess;
    }
    if (ok) ok = cudaMalloc(&mg->d_res, sizeof(double)) == cudaSuccess && cudaMallocHost(&mg->h_res, sizeof(double)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        mg_free(mg);
        return PB_ERR_NOMEM;
    }
    // Poisson form: the coarsest operator is known now; Helmholtz waits for alpha
    if (!is_helm(mg) && (e = setup_bottom(mg)) != PB_OK) {
        mg_free(mg);
        return e;
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
    if (!is_helm(mg)) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (is_mixed(mg)) {
        const int top = (int)mg->lv32.size() - 1;
        const long long n3 = (long long)mg->p.n * mg->p.n * mg->p.n;
        PB_CUDA(cudaMemcpyAsync(mg->alpha64, alpha, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
        k_to_float<<<grid_for(n3, 256), 256, 0, st>>>(mg->alpha64, mg->lv32[top].alpha, n3);
        PB_LAUNCH_CHECK();
        for (int l = top; l > 0; l--) {
            const long long nc3 = (long long)mg->lv32[l - 1].n * mg->lv32[l - 1].n * mg->lv32[l - 1].n;
            k_avgdown_plain<float><<<grid_for(nc3, 256), 256, 0, st>>>(mg->lv32[l].alpha, mg->lv32[l - 1].alpha, mg->lv32[l].n);
            PB_LAUNCH_CHECK();
        }
    } else {
        const int top = (int)mg->lv.size() - 1;
        MGLevel<double>& T = mg->lv[top];
        PB_CUDA(cudaMemcpyAsync(T.alpha, alpha, sizeof(double) * (size_t)T.n * T.n * T.n, cudaMemcpyDeviceToDevice, st));
        for (int l = top; l > 0; l--) {
            const long long nc3 = (long long)mg->lv[l - 1].n * mg->lv[l - 1].n * mg->lv[l - 1].n;
            k_avgdown_plain<double><<<grid_for(nc3, 256), 256, 0, st>>>(mg->lv[l].alpha, mg->lv[l - 1].alpha, mg->lv[l].n);
            PB_LAUNCH_CHECK();
        }
    }
    if (mg->p.bottom == PB_MG_BOTTOM_DIRECT) {
        PB_CUDA(cudaStreamSynchronize(st));
        return setup_bottom(mg);
    }
    return PB_OK;
}

int pb_mg_solve(pb_mg* mg, const double* rhs, double* phi, int* iters, double* hist, void* stream)
{
    if (!mg || !rhs || !phi) return PB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const bool mixed = is_mixed(mg);
    const int n = mg->p.n;
    const long long n3 = (long long)n * n * n;
    int e;
    MGLevel<double>* T = mixed ? nullptr : &mg->lv.back();
    if (mixed) {
        PB_CUDA(cudaMemcpyAsync(mg->f64, rhs, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
        k_pack_in<double><<<grid_for(n3, 256), 256, 0, st>>>(phi, mg->u64, n, grown_pitch<double>(n));
        PB_LAUNCH_CHECK();
        if ((e = launch_res64(mg, st)) != PB_OK) return e;
    } else {
        PB_CUDA(cudaMemcpyAsync(T->rhs, rhs, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
        T->cur = 0;
        k_pack_in<double><<<grid_for(n3, 256), 256, 0, st>>>(phi, T->phi[0], n, T->sx);
        PB_LAUNCH_CHECK();
        e = fuse_norm(mg) ? launch_relax_norm(mg, *T, st) : launch_resnorm(mg, *T, st);
        if (e != PB_OK) return e;
    }
    PB_CUDA(cudaMemcpyAsync(mg->h_res, mg->d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
    const double r0 = *mg->h_res;
    if (hist) hist[0] = r0;
    int it = 0;
    while (it < mg->p.max_iter) {
        // Replay the captured cycle when one exists for this state; capture it otherwise. The FP64
        // cycle flips the finest level's buffer nu1 + nu2 times, so it has one graph per parity;
        // the mixed cycle always starts from the same buffers.
        const int par = mixed ? 0 : T->cur;
        if (!mg->graph[par] && (it > 0 || mixed)) {
            if (!mg->graph_stream) PB_CUDA(cudaStreamCreateWithFlags(&mg->graph_stream, cudaStreamNonBlocking));
            cudaGraph_t g;
            PB_CUDA(cudaStreamBeginCapture(mg->graph_stream, cudaStreamCaptureModeThreadLocal));
            e = cycle_and_norm(mg, mg->graph_stream);
            cudaError_t ce = cudaStreamEndCapture(mg->graph_stream, &g);
            if (e != PB_OK) {
                if (ce == cudaSuccess) cudaGraphDestroy(g);
                return e;
            }
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            ce = cudaGraphInstantiate(&mg->graph[par], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            if (!mixed) {
                // capture recorded the buffer flips without running them
                mg->graph_cur[par] = T->cur;
                T->cur = par;
            }
        }
        if (mg->graph[par]) {
            PB_CUDA(cudaGraphLaunch(mg->graph[par], st));
            if (!mixed) T->cur = mg->graph_cur[par];
        } else {
            if ((e = cycle_and_norm(mg, st)) != PB_OK) return e;
        }
        PB_CUDA(cudaStreamSynchronize(st));
        const double r = *mg->h_res;
        ++it;
        if (hist) hist[it] = r;
        if (r < mg->p.tol * r0) break;
    }
    const double* src = mixed ? mg->u64 : T->phi[T->cur];
    k_pack_out<double><<<grid_for(n3, 256), 256, 0, st>>>(src, phi, n, grown_pitch<double>(n));
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaStreamSynchronize(st));
    if (read_error_mg() > 0 || read_error_stencil() > 0) return PB_ERR_DEVICE;
    if (iters) *iters = it;
    return PB_OK;
}

int pb_mg_solve_n(pb_mg* mg, const double* rhs, double* phi, int max_iter, double tol, int* iters, double* hist,
                  void* stream)
{
    if (!mg || max_iter < 0) return PB_ERR_ARG;
    const int keep_iter = mg->p.max_iter;
    const double keep_tol = mg->p.tol;
    mg->p.max_iter = max_iter;   // the captured cycles do not depend on either
    mg->p.tol = tol;
    const int e = pb_mg_solve(mg, rhs, phi, iters, hist, stream);
    mg->p.max_iter = keep_iter;
    mg->p.tol = keep_tol;
    return e;
}

int pb_mg_relax(pb_mg* mg, int sweeps, void* stream)
{
    if (!mg || sweeps < 0) return PB_ERR_ARG;
    if (is_mixed(mg)) return relax_sweeps(mg, mg->lv32.back(), sweeps, false, (cudaStream_t)stream);
    return relax_sweeps(mg, mg->lv.back(), sweeps, false, (cudaStream_t)stream);
}

int pb_mg_launches_per_cycle(const pb_mg_params* p)
{
    if (params_ok(p) != PB_OK) return -1;
    // mirrors cycle_and_norm / vcycle / relax_sweeps, counting kernel launches (memsets excluded)
    const pb_mg_params& q = *p;
    const int ft = fused_top(q);
    const int es = q.precision == PB_MG_MIXED ? 4 : 8;
    const bool helm = q.form == PB_MG_HELMHOLTZ;
    auto sweeps = [&](int n, int k, bool zero_start) {
        int s = 0, c = 0;
        if (zero_start && k >= 2 && relax2_edge(n, es, helm)) {
            s = 2;
            c = 1;
        } else if (zero_start && k > 0) {
            s = c = 1;
        }
        if (relax2_edge(n, es, helm))
            for (; s + 2 <= k; s += 2) c++;
        return c + (k - s);
    };
    std::function<int(int, bool, int, bool)> cyc = [&](int l, bool zero_start, int pre_done, bool fuse_update) {
        const int n = q.n >> (q.levels - l);
        if (zero_start && l == ft) return 1;
        if (l > 0) {
            int c = sweeps(n, q.nu1 - pre_done, zero_start && !pre_done) + 1 + cyc(l - 1, true, 0, false) + 1;
            if (!fuse_update) return c + sweeps(n, q.nu2, false);
            return c + (mixed_pairs(q) ? sweeps(n, q.nu2 - 2, false) : sweeps(n, q.nu2 - 1, false)) + 1;
        }
        return q.bottom == PB_MG_BOTTOM_DIRECT ? 1 : sweeps(n, q.nu_bottom, zero_start);
    };
    if (q.precision == PB_MG_MIXED) return (mixed_pairs(q) ? cyc(q.levels, true, 0, true) : cyc(q.levels, false, 1, true)) + 1;
    if (q.nu1 >= 1 && q.levels >= 1) return cyc(q.levels, false, norm_sweeps_for(q), false) + 1;
    return cyc(q.levels, false, 0, false) + 1;
}

int pb_mg_relax2_min_edge(int edge)
{
    if (edge < 0) return PB_ERR_ARG;
    g_relax2_min_edge = edge;
    return PB_OK;
}

int pb_mg_relax2_shape(int zc, int cells_per_thread, int rows_per_group)
{
    if (zc < 0 || cells_per_thread < 0 || cells_per_thread > 2) return PB_ERR_ARG;
    if (rows_per_group != 0 && rows_per_group != 2 && rows_per_group != 4) return PB_ERR_ARG;
    g_relax2_zc = zc;
    g_relax2_pv = cells_per_thread;
    g_relax2_rg = rows_per_group;
    return PB_OK;
}

int pb_mg_coarse_edge(int edge)
{
    if (edge < 0) return PB_ERR_ARG;
    g_coarse_edge = edge;
    return PB_OK;
}

} // extern "C"
