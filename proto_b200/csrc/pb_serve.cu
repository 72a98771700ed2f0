// Serving engine (C ABI: pb_serve_*): a stream of periodic Poisson/Helmholtz solves of different
// grid sizes, solved together. Each admitted solve keeps its hierarchy resident on the device (FP64
// solution and right-hand side, FP32 levels) for its whole life; admission is bounded by an HBM
// budget and a slot count. One step runs one mixed-precision V-cycle for every in-flight solve:
// each phase of the cycle (a sweep at one depth, a restriction, a prolongation, the coarse-level
// cycle, the FP64 residual pass) is one launch covering all solves, and the whole step is one CUDA
// graph, captured once per hierarchy depth and replayed while solves arrive and retire (the kernels
// read their work lists from device memory). Converged solves are copied out and their slots and
// memory reused.
//
// Per solve the arithmetic is the single-solve solver's of the engine's precision (pb_mg with
// PB_MG_MIXED or PB_MG_FP64, a constant alpha field, levels = the number of halvings, coarse levels
// of edge <= 16 fused), so a result is the same alone and in any mix, and the same as that solver's.
// The FP64 engine keeps every level in FP64: the top level is the solution itself, and each step
// ends with the residual norm fused with the first sweep of the next cycle, as the FP64 solver's
// norm pass; its results are those of the reference's own arithmetic.
//
// Reference counterpart: none (the reference runs one solve at a time, LevelMultigridSolver::solve,
// include/utils/implem/Proto_LevelMultigridSolverImplem.H:85-123).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "pb_internal.cuh"
#include "pb_serve_kernels.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

PB_DEFINE_ERROR_READER(read_error_serve)

// One device-resident hierarchy (reused across solves of the same edge).
struct SvHier {
    int n = 0;
    int nlev = 0;                       // levels, top first
    std::vector<int> edge, sx;          // per level
    // level buffers (FP32 levels of the mixed engine, FP64 levels of the FP64 engine); alpha: coarse
    // levels only (Helmholtz)
    std::vector<void*> phi0, phi1, rhs, alpha;
    double* u64 = nullptr;              // grown, pitch sxd (FP64 engine: the top level's phi[0])
    double* f64 = nullptr;              // n^3, also the staging buffer of the result (FP64 engine: the
                                        // top level's rho)
    int sxd = 0;
    size_t bytes = 0;
    void* slab = nullptr;               // one allocation holds every buffer above
};

struct SvSolve {
    long long ticket = 0;
    pb_serve_request req{};
    int state = PB_SERVE_WAITING;
    int slot = -1;
    SvHier* h = nullptr;
    int depth = 0;                      // batched levels (the top one and every edge > 16)
    std::vector<float> alpha_lv;        // per level: the FP32 alpha the single-solve solver has there
    std::vector<double> alpha_lv64;     // per level: the FP64 alpha (FP64 levels; [0] = the request's)
    int cycles = 0;
    double r0 = 0, r = 0;
    bool fresh = false;                 // admitted, first residual pass pending
};

} // namespace pb

using namespace pb;

struct pb_serve {
    pb_serve_params p{};
    bool fp64 = false;                  // every level in FP64 (PB_MG_FP64), else FP32 cycles
    int device = 0;
    cudaStream_t st = nullptr;
    long long next_ticket = 1;
    std::map<long long, SvSolve> solves;
    std::deque<long long> waiting;
    // admitted solves whose right-hand side is on its way to the device (upload stream); they take
    // a slot once it has landed, so uploads overlap the cycles of the solves already in flight
    struct Loading {
        long long ticket;
        cudaEvent_t landed;
    };
    std::deque<Loading> loading;
    std::vector<long long> slots;       // slot -> ticket (0: free)
    std::vector<long long> completed;   // tickets done since the last poll
    std::multimap<int, SvHier*> cache;  // idle hierarchies by edge
    // retired solves whose result is still on its way to the host (copy stream)
    struct Pending {
        long long ticket;
        SvHier* h;
        cudaEvent_t done;
        int state;                      // PB_SERVE_DONE / FAILED once the copy has landed
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> free_events;
    cudaStream_t cst = nullptr;         // copy stream for results
    cudaStream_t ust = nullptr;         // upload stream for admitted solves
    cudaMemPool_t pool = nullptr;       // device memory of the hierarchies
    size_t held = 0;                    // bytes of all hierarchies (busy and idle)
    // phase lists (device + host mirror)
    int max_phases = 0;
    SvItem* d_items = nullptr;
    long long* d_unit0 = nullptr;       // per phase: first rows of its items (compact, for the search)
    SvPhaseHeader* d_hdr = nullptr;
    // host mirrors in pinned memory (the copies to the device are asynchronous; each step ends with
    // a stream synchronisation, so a mirror is rebuilt only after its last copy has landed)
    SvItem* h_items = nullptr;
    long long* h_unit0 = nullptr;
    SvPhaseHeader* h_hdr = nullptr;
    void* d_cargs = nullptr;            // CoarseArgs<float> / CoarseArgs<double> per solve
    CoarseOffsets* d_coffs = nullptr;
    int* d_ccount = nullptr;
    void* h_cargs = nullptr;
    int* h_ccount = nullptr;
    CoarseOffsets* h_coffs = nullptr;
    double* d_norms = nullptr;          // per slot: residual norm of the step
    double* d_r0 = nullptr;             // per slot: first residual norm
    double* h_norms = nullptr;          // pinned
    double* h_r0 = nullptr;             // pinned
    // graphs by depth
    std::map<int, cudaGraphExec_t> graphs;
    bool lists_dirty = true;
    int depth_now = 0;
    int grid = 0;                       // persistent grid of the row-phase kernels
    int ring_grid = 0;                  // persistent grid of the staged kernels: every CTA resident
    size_t coarse_smem = 0;
    double t_stage[5] = {0, 0, 0, 0, 0};   // host seconds: admit, lists, residual pass, cycle, retire
    long long steps = 0;
};

namespace {

constexpr int kCoarseEdge = 16;
constexpr int kMaxDepth = 12;
// phases per depth (down: up to nu1 sweeps + restrict; up: prolong + nu2 sweeps) plus K1 slots
int phases_for(const pb_serve_params& p) { return kMaxDepth * (p.nu1 + p.nu2 + 2) + 2; }

bool edge_ok(int n)
{
    if (n < 2 || n % 2 != 0) return false;   // the top level is batched, so it must coarsen once
    int e = n;
    while (e > kCoarseEdge && e % 2 == 0) e /= 2;
    return e <= kCoarseEdge;
}

// Hierarchies come from the engine's own stream-ordered memory pool (release threshold = the HBM
// budget): freed slabs stay with the pool for later admissions, and neither allocating nor freeing
// waits for the device.
void hier_free(SvHier* h, cudaStream_t st)
{
    cudaFreeAsync(h->slab, st);
    delete h;
}

// Walks the buffers of an n-edge hierarchy in slab order (256-byte aligned offsets): per level the
// two grown solutions, rho and (edge <= 16) alpha, in the level type; then, for FP32 levels, the
// grown FP64 solution and the FP64 right-hand side. place(level, kind, offset, bytes) sees each;
// the return value is the slab size.
int level_pitch(int e, bool fp64) { return fp64 ? grown_pitch<double>(e) : grown_pitch<float>(e); }

template <class F>
size_t hier_layout(int n, bool fp64, F&& place)
{
    const size_t es = fp64 ? sizeof(double) : sizeof(float);
    size_t off = 0;
    auto put = [&](int l, int kind, size_t b) {
        place(l, kind, off, b);
        off += (b + 255) / 256 * 256;
    };
    int l = 0;
    for (int e = n;; e /= 2, l++) {
        const size_t g = es * (size_t)level_pitch(e, fp64) * (e + 2) * (e + 2);
        const size_t c = es * (size_t)e * e * e;
        put(l, 0, g);
        put(l, 1, g);
        put(l, 2, c);
        if (e <= kCoarseEdge) put(l, 3, c);
        if (e % 2 != 0 || e == 1) break;
    }
    if (!fp64) {
        put(-1, 4, sizeof(double) * (size_t)grown_pitch<double>(n) * (n + 2) * (n + 2));
        put(-1, 5, sizeof(double) * (size_t)n * n * n);
    }
    return off;
}

size_t hier_bytes(int n, bool fp64)
{
    return hier_layout(n, fp64, [](int, int, size_t, size_t) {});
}

// One allocation per hierarchy, ordered on stream st; the level solutions start at zero (their ghost
// images included), set on st as well.
SvHier* hier_alloc(int n, bool fp64, cudaMemPool_t pool, cudaStream_t st)
{
    SvHier* h = new SvHier;
    h->n = n;
    const size_t total = hier_bytes(n, fp64);
    if (cudaMallocFromPoolAsync(&h->slab, total, pool, st) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return nullptr;
    }
    unsigned char* base = static_cast<unsigned char*>(h->slab);
    bool ok = true;
    hier_layout(n, fp64, [&](int l, int kind, size_t off, size_t b) {
        if (l >= (int)h->edge.size()) {
            const int e = n >> l;
            h->edge.push_back(e);
            h->sx.push_back(level_pitch(e, fp64));
            h->phi0.push_back(nullptr);
            h->phi1.push_back(nullptr);
            h->rhs.push_back(nullptr);
            h->alpha.push_back(nullptr);
        }
        void* q = base + off;
        switch (kind) {
        case 0: h->phi0[l] = q; break;
        case 1: h->phi1[l] = q; break;
        case 2: h->rhs[l] = q; break;
        case 3: h->alpha[l] = q; break;
        case 4: h->u64 = static_cast<double*>(q); break;
        default: h->f64 = static_cast<double*>(q); break;
        }
        if (kind <= 1) ok = ok && cudaMemsetAsync(q, 0, b, st) == cudaSuccess;
    });
    h->nlev = (int)h->edge.size();
    h->sxd = grown_pitch<double>(n);
    if (fp64) {   // the top level is the FP64 solution and its right-hand side
        h->u64 = static_cast<double*>(h->phi0[0]);
        h->f64 = static_cast<double*>(h->rhs[0]);
    }
    h->bytes = total;
    if (!ok) {
        cudaGetLastError();
        hier_free(h, st);
        return nullptr;
    }
    return h;
}

bool make_pool(int device, size_t keep, cudaMemPool_t* out)
{
    cudaMemPoolProps pp;
    memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    if (cudaMemPoolCreate(out, &pp) != cudaSuccess) return false;
    uint64_t thr = keep;
    return cudaMemPoolSetAttribute(*out, cudaMemPoolAttrReleaseThreshold, &thr) == cudaSuccess;
}

int batched_depth(const SvHier* h)
{
    int d = 1;
    while (d < h->nlev && h->edge[d] > kCoarseEdge) d++;
    return d;
}

// Per-level FP32 alpha of a constant field: the top level holds float(alpha), each coarser level the
// 2^3 average of the one above (eight products 0.125*a summed in order, each rounded to FP32, as
// the averaging kernel does; for a non-dyadic a the sum is not exactly a).
template <typename T>
std::vector<T> level_alphas(double alpha, int nlev)
{
    std::vector<T> v(nlev);
    v[0] = (T)alpha;
    for (int l = 1; l < nlev; l++) {
        T acc = T(0);
        for (int k = 0; k < 8; k++) acc = acc + T(0.125) * v[l - 1];
        v[l] = acc;
    }
    return v;
}

// Smoother scalars of the level at depth d of an n-edge hierarchy (the single-solve solver's).
template <typename T>
RelaxCoef<T> level_coef(const pb_serve_params& p, const pb_serve_request& q, int n, int e, int sx, int d)
{
    const double h = (double)(1 << d) / (double)n, hsqinv = 1. / (h * h);
    RelaxCoef<T> k;
    k.n = e;
    k.sx = sx;
    k.helm = q.form == PB_MG_HELMHOLTZ;
    k.neg_lambda = (T)(-mg_lambda(p.omega, h));
    k.beta = (T)q.beta;
    k.omega = (T)p.omega;
    k.diagB = (T)(6.0 * q.beta * hsqinv);
    return k;
}

// units of the staged phases: 32 x 8 tiles x zd-deep z chunks, one CTA each
long long ring_units(int e, int zd)
{
    return (long long)((e + kSvTX - 1) / kSvTX) * ((e + kSvTY - 1) / kSvTY) * ((e + zd - 1) / zd);
}

double level_hsqinv(int n, int d)
{
    const double h = (double)(1 << d) / (double)n;
    return 1. / (h * h);
}

} // namespace

// ---- work lists ------------------------------------------------------------------------------------
// Phase order of one step (D = deepest batched depth among the active solves):
//   down d = 0..D-1 : sweeps (depth 0: nu1-1, the first ran in the residual pass; deeper: a sweep
//                     from zero then nu1-1), restriction to d+1
//   coarse          : the fused coarse cycle of every solve (one CTA each)
//   up d = D-1..0   : prolongation from d+1, sweeps (depth 0: nu2-1 then the fused update)
//   K1              : FP64 residual, norm, FP32 right-hand side and first sweep of the next step
// The FP64 engine's depth 0 is the solution itself: nu2 sweeps on the way up, and NORM (the residual
// norm with the first sweep of the next step) in K1's place.
// Phase slots are laid out in that order; the graph for depth D launches exactly these slots.
namespace {

struct PhaseSlot {
    int op;
    int depth;
};

std::vector<PhaseSlot> phase_plan(const pb_serve_params& p, int D)
{
    const bool fp64 = p.precision == PB_MG_FP64;
    std::vector<PhaseSlot> v;
    for (int d = 0; d < D; d++) {
        if (d == 0) {
            for (int s = 1; s < p.nu1; s++) v.push_back({SV_RELAX, d});
        } else {
            v.push_back({SV_RELAX_FIRST, d});
            for (int s = 1; s < p.nu1; s++) v.push_back({SV_RELAX, d});
        }
        v.push_back({SV_RESTRICT, d});
    }
    v.push_back({-1, -1});   // coarse
    for (int d = D - 1; d >= 0; d--) {
        v.push_back({SV_PROLONG, d});
        const int sweeps = d == 0 && !fp64 ? p.nu2 - 1 : p.nu2;
        for (int s = 0; s < sweeps; s++) v.push_back({SV_RELAX, d});
        if (d == 0 && !fp64) v.push_back({SV_UPDATE, 0});
    }
    v.push_back({fp64 ? SV_NORM : SV_K1, 0});
    return v;
}

// buffer index holding a level's current solution just before each phase, following the
// single-solve solver's ping-pong: depth 0 starts at 1 (the residual pass wrote phi[1]), deeper
// levels start from zero (their first sweep writes phi[1])
// Lays a phase's items out in unit order. Staged phases (a CTA per unit) take the deepest z chunk
// (32, 16, 8 or 4 planes) that still gives every CTA of the persistent grid a unit: deep chunks
// amortise the ring's fill, shallow ones keep a small batch from leaving most SMs idle. Row phases
// (a warp per row) round each item to whole CTAs.
long long layout_items(std::vector<SvItem>& items, bool staged, long long ctas)
{
    long long total = 0;
    if (staged) {
        int zd = 32;
        for (;; zd /= 2) {
            long long sum = 0;
            for (const SvItem& it : items) sum += ring_units(it.k.n, zd);
            if (sum >= ctas || zd <= 4) break;
        }
        for (SvItem& it : items) {
            it.zd = zd;
            it.units = (int)ring_units(it.k.n, zd);
            it.unit0 = total;
            total += it.units;
        }
        return total;
    }
    for (SvItem& it : items) {
        it.unit0 = total;
        total += ((long long)it.units + kSvRows - 1) / kSvRows * kSvRows;
    }
    return total;
}

bool is_staged(int op) { return op == SV_RELAX || op == SV_UPDATE || op == SV_K1 || op == SV_NORM; }

// The fields of an item at depth d of solve s that every phase shares: geometry and smoother scalars
// (FP32 always: the geometry of the work layout; FP64 for FP64 levels), alpha and beta, the slot and
// the FP64 top-level buffers.
SvItem item_base(const pb_serve_params& p, bool fp64, const SvSolve& s, int d)
{
    const SvHier& h = *s.h;
    SvItem it{};
    it.k = level_coef<float>(p, s.req, h.n, h.edge[d], h.sx[d], d);
    if (fp64) it.k64 = level_coef<double>(p, s.req, h.n, h.edge[d], h.sx[d], d);
    it.alpha = s.alpha_lv[d];
    it.beta = (float)s.req.beta;
    it.alpha64 = s.alpha_lv64[d];
    it.beta64 = s.req.beta;
    it.slot = s.slot;
    it.sxd = h.sxd;
    it.u64 = h.u64;
    it.f64 = h.f64;
    return it;
}

// the 7-point coefficients scaled by sc, in the item's level type(s)
void item_coefs(SvItem& it, bool fp64, double sc)
{
    it.c = lap7_coefs<float>(sc);
    if (fp64) it.c64 = lap7_coefs<double>(sc);
}

// the FP64 engine's norm pass over the top level: state in phi[0], first sweep into phi[1]
SvItem norm_item(const pb_serve_params& p, const SvSolve& s)
{
    const SvHier& h = *s.h;
    const bool helm = s.req.form == PB_MG_HELMHOLTZ;
    SvItem it = item_base(p, true, s, 0);
    it.in = h.phi0[0];
    it.out = h.phi1[0];
    it.rhs = h.rhs[0];
    const double hs = level_hsqinv(h.n, 0);
    item_coefs(it, true, helm ? hs : p.omega / 6.0);
    it.nscale = hs;
    return it;
}

} // namespace

template <typename T>
static int fill_coarse_args(pb_serve* sv, const std::vector<SvSolve*>& act)
{
    const pb_serve_params& p = sv->p;
    const int cap = (int)p.max_active;
    CoarseArgs<T>* hc = static_cast<CoarseArgs<T>*>(sv->h_cargs);
    memset(hc, 0, sizeof(CoarseArgs<T>) * cap);
    memset(sv->h_coffs, 0, sizeof(CoarseOffsets) * cap);
    int nc = 0;
    for (size_t a = 0; a < act.size(); a++) {
        SvSolve& s = *act[a];
        SvHier& h = *s.h;
        CoarseArgs<T> ca;
        memset(&ca, 0, sizeof(ca));
        const int d0 = s.depth, top = h.nlev - 1 - d0;   // coarse levels: index 0 = coarsest
        const bool helm = s.req.form == PB_MG_HELMHOLTZ;
        for (int l = 0; l <= top; l++) {
            const int d = h.nlev - 1 - l;
            CoarseLevel<T>& c = ca.lv[l];
            c.phi[0] = static_cast<T*>(h.phi0[d]);
            c.phi[1] = static_cast<T*>(h.phi1[d]);
            c.rhs = static_cast<T*>(h.rhs[d]);
            c.alpha = static_cast<const T*>(h.alpha[d]);
            c.k = level_coef<T>(p, s.req, h.n, h.edge[d], h.sx[d], d);
            const double hs = level_hsqinv(h.n, d);
            c.crelax = lap7_coefs<T>(helm ? hs : p.omega / 6.0);
            c.cres = lap7_coefs<T>(helm ? hs : -hs);
        }
        ca.top = top;
        ca.nu1 = p.nu1;
        ca.nu2 = p.nu2;
        ca.nu_bottom = p.nu_bottom;
        ca.direct = 0;
        ca.ainv = nullptr;
        ca.beta = (T)s.req.beta;
        CoarseOffsets off;
        memset(&off, 0, sizeof(off));
        const size_t smem = coarse_smem_layout(ca, helm, off.o);
        ca.in_smem = smem <= sv->coarse_smem ? 1 : 0;
        hc[nc] = ca;
        sv->h_coffs[nc] = off;
        nc++;
    }
    PB_CUDA(cudaMemcpyAsync(sv->d_cargs, sv->h_cargs, sizeof(CoarseArgs<T>) * nc, cudaMemcpyHostToDevice, sv->st));
    PB_CUDA(cudaMemcpyAsync(sv->d_coffs, sv->h_coffs, sizeof(CoarseOffsets) * nc, cudaMemcpyHostToDevice, sv->st));
    *sv->h_ccount = nc;
    PB_CUDA(cudaMemcpyAsync(sv->d_ccount, sv->h_ccount, sizeof(int), cudaMemcpyHostToDevice, sv->st));
    return PB_OK;
}

static int build_lists(pb_serve* sv)
{
    const pb_serve_params& p = sv->p;
    const bool fp64 = sv->fp64;
    int D = 0;
    std::vector<SvSolve*> act;
    for (long long t : sv->slots)
        if (t) {
            SvSolve& s = sv->solves[t];
            act.push_back(&s);
            D = std::max(D, s.depth);
        }
    sv->depth_now = D;
    const std::vector<PhaseSlot> plan = phase_plan(p, std::max(D, 1));
    const int cap = (int)p.max_active;
    for (int ph = 0; ph < sv->max_phases; ph++) sv->h_hdr[ph] = SvPhaseHeader{0, 0};
    // per solve: the buffer index of each level's current solution as the plan advances
    std::vector<std::vector<int>> cur(act.size());
    for (size_t a = 0; a < act.size(); a++) {
        cur[a].assign(act[a]->h->nlev, 0);
        cur[a][0] = 1;
    }
    for (size_t ph = 0; ph < plan.size(); ph++) {
        const PhaseSlot& ps = plan[ph];
        if (ps.op < 0) continue;   // coarse: its own argument table
        std::vector<SvItem> items;
        for (size_t a = 0; a < act.size(); a++) {
            SvSolve& s = *act[a];
            SvHier& h = *s.h;
            const int d = ps.depth;
            if (d >= s.depth) continue;
            const int n = h.n, e = h.edge[d];
            SvItem it = item_base(p, fp64, s, d);
            const bool helm = s.req.form == PB_MG_HELMHOLTZ;
            void* ph_[2] = {h.phi0[d], h.phi1[d]};
            int& c = cur[a][d];
            switch (ps.op) {
            case SV_RELAX:
            case SV_UPDATE:
                it.in = ph_[c];
                it.out = ph_[1 - c];
                it.rhs = h.rhs[d];
                item_coefs(it, fp64, helm ? level_hsqinv(n, d) : p.omega / 6.0);
                if (ps.op == SV_RELAX) c = 1 - c;
                break;
            case SV_RELAX_FIRST:
                c = 0;
                it.out = ph_[1];
                it.rhs = h.rhs[d];
                it.units = e * e;
                c = 1;
                break;
            case SV_RESTRICT: {
                it.in = ph_[c];
                it.out = h.rhs[d + 1];
                it.rhs = h.rhs[d];
                const double hs = level_hsqinv(n, d);
                item_coefs(it, fp64, helm ? hs : -hs);
                it.units = (e / 2) * (e / 2);
                break;
            }
            case SV_PROLONG: {
                it.in = ph_[c];
                const int dc = d + 1;
                // the coarse part leaves its entry level's result in phi[0]
                const int cc = dc >= s.depth ? 0 : cur[a][dc];
                it.delta = cc ? h.phi1[dc] : h.phi0[dc];
                it.sxc = h.sx[dc];
                it.units = e * e;
                break;
            }
            case SV_K1: {
                it.in = h.phi1[0];
                it.out = h.rhs[0];
                const double hs = level_hsqinv(n, 0);
                it.c64 = lap7_coefs<double>(helm ? hs : -hs);
                c = 1;
                break;
            }
            case SV_NORM:
                // the cycle's sweeps come back to phi[0] (nu1 + nu2 is even)
                it = norm_item(p, s);
                c = 1;
                break;
            }
            items.push_back(it);
        }
        const long long total = layout_items(items, is_staged(ps.op), is_staged(ps.op) ? sv->ring_grid : sv->grid);
        std::copy(items.begin(), items.end(), sv->h_items + ph * cap);
        for (size_t k = 0; k < items.size(); k++) sv->h_unit0[ph * cap + k] = items[k].unit0;
        sv->h_hdr[ph] = SvPhaseHeader{(long long)items.size(), total};
    }
    // the residual pass for freshly admitted solves (slot max_phases-1)
    {
        const int ph = sv->max_phases - 1;
        std::vector<SvItem> items;
        for (size_t a = 0; a < act.size(); a++) {
            SvSolve& s = *act[a];
            if (!s.fresh) continue;
            if (fp64) {
                items.push_back(norm_item(p, s));
                continue;
            }
            SvHier& h = *s.h;
            const bool helm = s.req.form == PB_MG_HELMHOLTZ;
            SvItem it = item_base(p, false, s, 0);
            it.in = h.phi1[0];
            it.out = h.rhs[0];
            const double hs = level_hsqinv(h.n, 0);
            it.c64 = lap7_coefs<double>(helm ? hs : -hs);
            items.push_back(it);
        }
        const long long total = layout_items(items, true, sv->ring_grid);
        std::copy(items.begin(), items.end(), sv->h_items + (size_t)ph * cap);
        for (size_t k = 0; k < items.size(); k++) sv->h_unit0[(size_t)ph * cap + k] = items[k].unit0;
        sv->h_hdr[ph] = SvPhaseHeader{(long long)items.size(), total};
    }
    // the phases of this depth's plan and the residual-pass slot (the last one)
    const size_t used = plan.size() * cap;
    PB_CUDA(cudaMemcpyAsync(sv->d_items, sv->h_items, sizeof(SvItem) * used, cudaMemcpyHostToDevice, sv->st));
    PB_CUDA(cudaMemcpyAsync(sv->d_unit0, sv->h_unit0, sizeof(long long) * used, cudaMemcpyHostToDevice, sv->st));
    const size_t last = (size_t)(sv->max_phases - 1) * cap;
    PB_CUDA(cudaMemcpyAsync(sv->d_items + last, sv->h_items + last, sizeof(SvItem) * cap, cudaMemcpyHostToDevice, sv->st));
    PB_CUDA(cudaMemcpyAsync(sv->d_unit0 + last, sv->h_unit0 + last, sizeof(long long) * cap, cudaMemcpyHostToDevice, sv->st));
    PB_CUDA(cudaMemcpyAsync(sv->d_hdr, sv->h_hdr, sizeof(SvPhaseHeader) * sv->max_phases, cudaMemcpyHostToDevice, sv->st));
    // coarse-cycle arguments (entry level = depth s.depth)
    const int e = fp64 ? fill_coarse_args<double>(sv, act) : fill_coarse_args<float>(sv, act);
    if (e != PB_OK) return e;
    sv->lists_dirty = false;
    return PB_OK;
}

static int launch_phase(pb_serve* sv, int slot, int op, double* norms, cudaStream_t st)
{
    const SvItem* items = sv->d_items + (size_t)slot * sv->p.max_active;
    const long long* u0 = sv->d_unit0 + (size_t)slot * sv->p.max_active;
    const SvPhaseHeader* hdr = sv->d_hdr + slot;
    const int rg = sv->ring_grid, g = sv->grid;
    if (sv->fp64) {
        switch (op) {
        case SV_RELAX: k_sv_ring<SV_RELAX, double><<<rg, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_RELAX_FIRST: k_sv_phase<SV_RELAX_FIRST, double><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_RESTRICT: k_sv_phase<SV_RESTRICT, double><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_PROLONG: k_sv_phase<SV_PROLONG, double><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_NORM: k_sv_ring<SV_NORM, double><<<rg, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        default: return PB_ERR_ARG;
        }
    } else {
        switch (op) {
        case SV_RELAX: k_sv_ring<SV_RELAX, float><<<rg, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_RELAX_FIRST: k_sv_phase<SV_RELAX_FIRST, float><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_RESTRICT: k_sv_phase<SV_RESTRICT, float><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_PROLONG: k_sv_phase<SV_PROLONG, float><<<g, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_K1: k_sv_ring<SV_K1, double><<<rg, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        case SV_UPDATE: k_sv_ring<SV_UPDATE, float><<<rg, kSvUnit, 0, st>>>(items, u0, hdr, norms); break;
        default: return PB_ERR_ARG;
        }
    }
    PB_LAUNCH_CHECK();
    return PB_OK;
}

// One step's work for depth D, in stream order (captured into a graph).
static int enqueue_step(pb_serve* sv, int D, cudaStream_t st)
{
    const std::vector<PhaseSlot> plan = phase_plan(sv->p, D);
    int e;
    for (size_t ph = 0; ph < plan.size(); ph++) {
        const PhaseSlot& ps = plan[ph];
        if (ps.op < 0) {
            if (sv->fp64)
                k_coarse_cycle_batch<double><<<sv->p.max_active, kCoarseThreads, sv->coarse_smem, st>>>(
                    static_cast<const CoarseArgs<double>*>(sv->d_cargs), sv->d_coffs, sv->d_ccount);
            else
                k_coarse_cycle_batch<float><<<sv->p.max_active, kCoarseThreads, sv->coarse_smem, st>>>(
                    static_cast<const CoarseArgs<float>*>(sv->d_cargs), sv->d_coffs, sv->d_ccount);
            PB_LAUNCH_CHECK();
            continue;
        }
        if (ps.op == SV_K1 || ps.op == SV_NORM) PB_CUDA(cudaMemsetAsync(sv->d_norms, 0, sizeof(double) * sv->p.max_active, st));
        if ((e = launch_phase(sv, (int)ph, ps.op, sv->d_norms, st)) != PB_OK) return e;
    }
    PB_CUDA(cudaMemcpyAsync(sv->h_norms, sv->d_norms, sizeof(double) * sv->p.max_active, cudaMemcpyDeviceToHost, st));
    return PB_OK;
}

static cudaEvent_t take_event(pb_serve* sv)
{
    if (sv->free_events.empty()) {
        for (int k = 0; k < 8; k++) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
            sv->free_events.push_back(e);
        }
    }
    cudaEvent_t e = sv->free_events.back();
    sv->free_events.pop_back();
    return e;
}

// Admission, in request order, while the HBM budget allows and fewer than max(2, max_active / 4)
// solves are loading (a few steps' worth of retirements: more would only hold hierarchies idle):
// the solve takes a hierarchy (a cached one of its edge, else a new one, dropping idle
// hierarchies of other edges to make room) and its right-hand side goes up on the upload stream.
static int admit(pb_serve* sv)
{
    const int max_loading = std::max(2, sv->p.max_active / 4);
    while (!sv->waiting.empty() && (int)sv->loading.size() < max_loading) {
        SvSolve& s = sv->solves[sv->waiting.front()];
        const int n = s.req.n;
        SvHier* h = nullptr;
        auto it = sv->cache.find(n);
        if (it != sv->cache.end()) {
            h = it->second;
            sv->cache.erase(it);
        } else {
            const size_t need = hier_bytes(n, sv->fp64);
            // make room by dropping idle hierarchies of other edges
            while (sv->held + need > (size_t)sv->p.hbm_budget && !sv->cache.empty()) {
                auto v = sv->cache.begin();
                sv->held -= v->second->bytes;
                hier_free(v->second, sv->ust);
                sv->cache.erase(v);
            }
            if (sv->held + need > (size_t)sv->p.hbm_budget) return PB_OK;   // wait for memory
            h = hier_alloc(n, sv->fp64, sv->pool, sv->ust);
            if (!h) return PB_OK;
            sv->held += h->bytes;
        }
        cudaEvent_t landed = take_event(sv);
        if (!landed) {
            sv->cache.insert({n, h});
            return PB_ERR_CUDA;
        }
        sv->waiting.pop_front();
        s.h = h;
        s.state = PB_SERVE_ACTIVE;
        s.depth = batched_depth(h);
        s.alpha_lv = level_alphas<float>(s.req.alpha, h->nlev);
        s.alpha_lv64 = level_alphas<double>(s.req.alpha, h->nlev);
        // initial guess zero, right-hand side in; constant alpha on the coarse levels
        const size_t n3 = (size_t)n * n * n;
        PB_CUDA(cudaMemsetAsync(h->u64, 0, sizeof(double) * (size_t)h->sxd * (n + 2) * (n + 2), sv->ust));
        PB_CUDA(cudaMemcpyAsync(h->f64, s.req.rhs, sizeof(double) * n3, cudaMemcpyHostToDevice, sv->ust));
        if (s.req.form == PB_MG_HELMHOLTZ)
            for (int d = 0; d < h->nlev; d++)
                if (h->alpha[d]) {
                    const long long c = (long long)h->edge[d] * h->edge[d] * h->edge[d];
                    if (sv->fp64)
                        k_sv_fill<double><<<grid_for(c, 256), 256, 0, sv->ust>>>(static_cast<double*>(h->alpha[d]), c,
                                                                                 s.alpha_lv64[d]);
                    else
                        k_sv_fill<float><<<grid_for(c, 256), 256, 0, sv->ust>>>(static_cast<float*>(h->alpha[d]), c,
                                                                               s.alpha_lv[d]);
                    PB_LAUNCH_CHECK();
                }
        PB_CUDA(cudaEventRecord(landed, sv->ust));
        sv->loading.push_back({s.ticket, landed});
    }
    return PB_OK;
}

// Loaded solves take free slots in admission order. Under a backlog (requests still queued) a solve
// whose upload has not landed waits for the next step, so uploads overlap the running cycles; with
// no backlog, or nothing in flight, the upload is waited for and the solve joins this step (light
// load: latency first).
static int join(pb_serve* sv)
{
    bool any = false;
    for (long long t : sv->slots) any = any || t;
    const bool backlog = !sv->waiting.empty();
    while (!sv->loading.empty()) {
        int slot = -1;
        for (int i = 0; i < (int)sv->slots.size(); i++)
            if (!sv->slots[i]) {
                slot = i;
                break;
            }
        if (slot < 0) return PB_OK;
        const pb_serve::Loading q = sv->loading.front();
        cudaError_t r = (any && backlog) ? cudaEventQuery(q.landed) : cudaEventSynchronize(q.landed);
        if (r == cudaErrorNotReady) return PB_OK;
        if (r != cudaSuccess) { set_cuda_error(r); return PB_ERR_CUDA; }
        sv->loading.pop_front();
        sv->free_events.push_back(q.landed);
        SvSolve& s = sv->solves[q.ticket];
        s.slot = slot;
        s.fresh = true;
        sv->slots[slot] = s.ticket;
        sv->lists_dirty = true;
        any = true;
    }
    return PB_OK;
}

// A finished solve leaves the cycle at once; its result goes to the host on the copy stream, and the
// ticket is reported (and the hierarchy reused) when that copy has landed.
static int retire(pb_serve* sv, SvSolve& s, int state)
{
    SvHier* h = s.h;
    const int n = h->n;
    const size_t n3 = (size_t)n * n * n;
    cudaEvent_t packed = take_event(sv);
    cudaEvent_t done = packed ? take_event(sv) : nullptr;
    if (!done) {
        if (packed) sv->free_events.push_back(packed);
        return PB_ERR_CUDA;
    }
    k_sv_pack_out<<<grid_for((long long)n3, 256), 256, 0, sv->st>>>(h->u64, h->f64, n, h->sxd);
    PB_LAUNCH_CHECK();
    PB_CUDA(cudaEventRecord(packed, sv->st));
    PB_CUDA(cudaStreamWaitEvent(sv->cst, packed, 0));
    PB_CUDA(cudaMemcpyAsync(s.req.out, h->f64, sizeof(double) * n3, cudaMemcpyDeviceToHost, sv->cst));
    PB_CUDA(cudaEventRecord(done, sv->cst));
    sv->free_events.push_back(packed);   // reusable once recorded again later (stream order keeps it valid)
    sv->slots[s.slot] = 0;
    s.slot = -1;
    s.h = nullptr;
    sv->pending.push_back({s.ticket, h, done, state});
    sv->lists_dirty = true;
    return PB_OK;
}

// Moves landed results to the completed list and their hierarchies to the cache; wait = block.
static int drain(pb_serve* sv, bool wait)
{
    if (wait && !sv->pending.empty()) PB_CUDA(cudaStreamSynchronize(sv->cst));
    for (size_t k = 0; k < sv->pending.size();) {
        auto& q = sv->pending[k];
        const cudaError_t r = cudaEventQuery(q.done);
        if (r == cudaErrorNotReady) {
            k++;
            continue;
        }
        if (r != cudaSuccess) { set_cuda_error(r); return PB_ERR_CUDA; }
        sv->cache.insert({q.h->n, q.h});
        sv->solves[q.ticket].state = q.state;
        sv->completed.push_back(q.ticket);
        sv->free_events.push_back(q.done);
        sv->pending.erase(sv->pending.begin() + k);
    }
    return PB_OK;
}

extern "C" {

int pb_serve_create(const pb_serve_params* p, pb_serve** out)
{
    if (!p || !out) return PB_ERR_ARG;
    if (p->max_active < 1 || p->max_active > kSvMaxSolves || p->nu1 < 1 || p->nu2 < 1 || p->nu_bottom < 0 ||
        p->hbm_budget <= 0 || !(p->tol > 0) || p->max_cycles < 1)
        return PB_ERR_ARG;
    if (p->precision != PB_MG_MIXED && p->precision != PB_MG_FP64) return PB_ERR_ARG;
    // FP64: each cycle's sweeps of the top level return to the buffer the norm pass reads
    if (p->precision == PB_MG_FP64 && (p->nu1 + p->nu2) % 2 != 0) return PB_ERR_ARG;
    pb_serve* sv = new (std::nothrow) pb_serve;
    if (!sv) return PB_ERR_NOMEM;
    sv->p = *p;
    sv->fp64 = p->precision == PB_MG_FP64;
    cudaGetDevice(&sv->device);
    sv->slots.assign(p->max_active, 0);
    sv->max_phases = phases_for(*p);
    const size_t cap = (size_t)p->max_active;
    bool ok = cudaStreamCreateWithFlags(&sv->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&sv->cst, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&sv->ust, cudaStreamNonBlocking) == cudaSuccess &&
              make_pool(sv->device, (size_t)p->hbm_budget, &sv->pool) &&
              cudaMallocHost(&sv->h_items, sizeof(SvItem) * cap * sv->max_phases) == cudaSuccess &&
              cudaMallocHost(&sv->h_unit0, sizeof(long long) * cap * sv->max_phases) == cudaSuccess &&
              cudaMallocHost(&sv->h_hdr, sizeof(SvPhaseHeader) * sv->max_phases) == cudaSuccess &&
              cudaMallocHost(&sv->h_cargs, sizeof(CoarseArgs<double>) * cap) == cudaSuccess &&
              cudaMallocHost(&sv->h_coffs, sizeof(CoarseOffsets) * cap) == cudaSuccess &&
              cudaMallocHost(&sv->h_ccount, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&sv->d_items, sizeof(SvItem) * cap * sv->max_phases) == cudaSuccess &&
              cudaMalloc(&sv->d_unit0, sizeof(long long) * cap * sv->max_phases) == cudaSuccess &&
              cudaMalloc(&sv->d_hdr, sizeof(SvPhaseHeader) * sv->max_phases) == cudaSuccess &&
              cudaMalloc(&sv->d_cargs, sizeof(CoarseArgs<double>) * cap) == cudaSuccess &&
              cudaMalloc(&sv->d_coffs, sizeof(CoarseOffsets) * cap) == cudaSuccess &&
              cudaMalloc(&sv->d_ccount, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&sv->d_norms, sizeof(double) * cap) == cudaSuccess &&
              cudaMalloc(&sv->d_r0, sizeof(double) * cap) == cudaSuccess &&
              cudaMallocHost(&sv->h_norms, sizeof(double) * cap) == cudaSuccess &&
              cudaMallocHost(&sv->h_r0, sizeof(double) * cap) == cudaSuccess;
    if (ok) {
        sv->grid = cached_sm_count() * 8;
        // the staged kernels take whole units per CTA: a grid of exactly the resident CTAs spreads
        // the units evenly (a larger one would run in partial waves)
        int o1 = 0, o2 = 0, o3 = 0;
        if (sv->fp64) {
            ok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_sv_ring<SV_RELAX, double>, kSvUnit, 0) == cudaSuccess &&
                 cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_sv_ring<SV_NORM, double>, kSvUnit, 0) == cudaSuccess;
            o3 = o1;
        } else {
            ok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_sv_ring<SV_RELAX, float>, kSvUnit, 0) == cudaSuccess &&
                 cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_sv_ring<SV_K1, double>, kSvUnit, 0) == cudaSuccess &&
                 cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, k_sv_ring<SV_UPDATE, float>, kSvUnit, 0) == cudaSuccess;
        }
        sv->ring_grid = cached_sm_count() * std::max(1, std::min(o1, std::min(o2, o3)));
        // coarse part: the largest arena (edge 16, Helmholtz) in shared memory where it fits (FP32
        // levels); otherwise the solves whose arena fits use shared memory and the rest global memory
        int l = 0;
        for (int e = kCoarseEdge; e >= 1; e /= 2, l++) {}
        auto arena = [&](auto zero) {
            using T = decltype(zero);
            CoarseArgs<T> ca;
            memset(&ca, 0, sizeof(ca));
            ca.top = l - 1;
            for (int i = 0, e = 1; i < l; i++, e *= 2) {
                ca.lv[i].k.n = e;
                ca.lv[i].k.sx = grown_pitch<T>(e);
            }
            return coarse_smem_layout(ca, 1, nullptr);
        };
        // the descriptor table takes a little static shared memory beside the arena
        sv->coarse_smem = std::min(sv->fp64 ? arena(0.0) : arena(0.f), (size_t)216 * 1024);
        if (sv->fp64)
            ok = ok && cudaFuncSetAttribute(k_coarse_cycle_batch<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sv->coarse_smem) == cudaSuccess;
        else
            ok = ok && cudaFuncSetAttribute(k_coarse_cycle_batch<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sv->coarse_smem) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        pb_serve_destroy(sv);
        return PB_ERR_NOMEM;
    }
    *out = sv;
    return PB_OK;
}

int pb_serve_destroy(pb_serve* sv)
{
    if (!sv) return PB_OK;
    if (sv->st) cudaStreamSynchronize(sv->st);
    if (sv->cst) cudaStreamSynchronize(sv->cst);
    if (sv->ust) cudaStreamSynchronize(sv->ust);
    for (auto& q : sv->loading) cudaEventDestroy(q.landed);
    for (auto& q : sv->pending) {
        hier_free(q.h, sv->ust);
        cudaEventDestroy(q.done);
    }
    for (cudaEvent_t e : sv->free_events) cudaEventDestroy(e);
    for (auto& g : sv->graphs) cudaGraphExecDestroy(g.second);
    for (auto& s : sv->solves)
        if (s.second.h) hier_free(s.second.h, sv->ust);
    for (auto& c : sv->cache) hier_free(c.second, sv->ust);
    if (sv->ust) cudaStreamSynchronize(sv->ust);
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    cudaFree(sv->d_items);
    cudaFree(sv->d_unit0);
    cudaFree(sv->d_hdr);
    cudaFree(sv->d_cargs);
    cudaFree(sv->d_coffs);
    cudaFree(sv->d_ccount);
    cudaFree(sv->d_norms);
    cudaFree(sv->d_r0);
    cudaFreeHost(sv->h_norms);
    cudaFreeHost(sv->h_r0);
    cudaFreeHost(sv->h_items);
    cudaFreeHost(sv->h_unit0);
    cudaFreeHost(sv->h_hdr);
    cudaFreeHost(sv->h_cargs);
    cudaFreeHost(sv->h_coffs);
    cudaFreeHost(sv->h_ccount);
    if (sv->st) cudaStreamDestroy(sv->st);
    if (sv->cst) cudaStreamDestroy(sv->cst);
    if (sv->ust) cudaStreamDestroy(sv->ust);
    delete sv;
    return PB_OK;
}

int pb_serve_submit(pb_serve* sv, const pb_serve_request* q, long long* ticket)
{
    if (!sv || !q || !q->rhs || !q->out) return PB_ERR_ARG;
    if (!edge_ok(q->n) || (q->form != PB_MG_POISSON && q->form != PB_MG_HELMHOLTZ)) return PB_ERR_ARG;
    if (hier_bytes(q->n, sv->fp64) > (size_t)sv->p.hbm_budget) return PB_ERR_BUDGET;
    SvSolve s;
    s.ticket = sv->next_ticket++;
    s.req = *q;
    if (s.req.form == PB_MG_POISSON) {
        s.req.alpha = 0.0;
        s.req.beta = 1.0;
    }
    sv->solves[s.ticket] = s;
    sv->waiting.push_back(s.ticket);
    if (ticket) *ticket = s.ticket;
    return PB_OK;
}

int pb_serve_step(pb_serve* sv, int* active, int* waiting)
{
    if (!sv) return PB_ERR_ARG;
    using clk = std::chrono::steady_clock;
    auto lap = [](clk::time_point& t0) {
        const clk::time_point t1 = clk::now();
        const double s = std::chrono::duration<double>(t1 - t0).count();
        t0 = t1;
        return s;
    };
    clk::time_point t0 = clk::now();
    int e;
    if ((e = drain(sv, false)) != PB_OK) return e;
    if ((e = admit(sv)) != PB_OK) return e;
    if ((e = join(sv)) != PB_OK) return e;
    sv->t_stage[0] += lap(t0);
    bool any = false;
    for (long long t : sv->slots) any = any || t;
    if (any) {
        sv->steps++;
        if (sv->lists_dirty && (e = build_lists(sv)) != PB_OK) return e;
        sv->t_stage[1] += lap(t0);
        // first residual pass of the solves admitted since the last step
        bool fresh = false;
        for (long long t : sv->slots)
            if (t && sv->solves[t].fresh) fresh = true;
        if (fresh) {
            PB_CUDA(cudaMemsetAsync(sv->d_r0, 0, sizeof(double) * sv->p.max_active, sv->st));
            if ((e = launch_phase(sv, sv->max_phases - 1, sv->fp64 ? SV_NORM : SV_K1, sv->d_r0, sv->st)) != PB_OK) return e;
            PB_CUDA(cudaMemcpyAsync(sv->h_r0, sv->d_r0, sizeof(double) * sv->p.max_active, cudaMemcpyDeviceToHost, sv->st));
        }
        sv->t_stage[2] += lap(t0);
        const int D = std::max(sv->depth_now, 1);
        auto g = sv->graphs.find(D);
        if (g == sv->graphs.end()) {
            cudaGraph_t graph;
            PB_CUDA(cudaStreamBeginCapture(sv->st, cudaStreamCaptureModeThreadLocal));
            e = enqueue_step(sv, D, sv->st);
            cudaError_t ce = cudaStreamEndCapture(sv->st, &graph);
            if (e != PB_OK) {
                if (ce == cudaSuccess) cudaGraphDestroy(graph);
                return e;
            }
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            cudaGraphExec_t ex;
            ce = cudaGraphInstantiate(&ex, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) { set_cuda_error(ce); return PB_ERR_CUDA; }
            g = sv->graphs.insert({D, ex}).first;
        }
        PB_CUDA(cudaGraphLaunch(g->second, sv->st));
        PB_CUDA(cudaStreamSynchronize(sv->st));
        sv->t_stage[3] += lap(t0);
        if (read_error_serve() > 0) return PB_ERR_DEVICE;
        // bookkeeping: converged or out of cycles -> copy out and free the slot
        for (int i = 0; i < (int)sv->slots.size(); i++) {
            const long long t = sv->slots[i];
            if (!t) continue;
            SvSolve& s = sv->solves[t];
            if (s.fresh) {
                s.r0 = sv->h_r0[i];
                s.fresh = false;
                sv->lists_dirty = true;
            }
            s.cycles++;
            s.r = sv->h_norms[i];
            // a residual that is not finite (a NaN or infinite right-hand side, or a diverging
            // solve) ends the solve at once as failed; its neighbours in the batch are unaffected
            if (!std::isfinite(s.r0) || !std::isfinite(s.r)) e = retire(sv, s, PB_SERVE_FAILED);
            else if (s.r < sv->p.tol * s.r0) e = retire(sv, s, PB_SERVE_DONE);
            else if (s.cycles >= sv->p.max_cycles) e = retire(sv, s, PB_SERVE_FAILED);
            if (e != PB_OK) return e;
        }
        sv->t_stage[4] += lap(t0);
    } else if ((e = drain(sv, true)) != PB_OK) {   // nothing in flight: deliver what is on its way
        return e;
    }
    int na = (int)sv->pending.size();
    for (long long t : sv->slots) na += t ? 1 : 0;
    if (active) *active = na;
    if (waiting) *waiting = (int)(sv->waiting.size() + sv->loading.size());
    return PB_OK;
}

int pb_serve_poll(pb_serve* sv, long long* tickets, int cap, int* n)
{
    if (!sv || !n || (cap > 0 && !tickets)) return PB_ERR_ARG;
    const int e = drain(sv, false);
    if (e != PB_OK) return e;
    const int k = std::min(cap, (int)sv->completed.size());
    for (int i = 0; i < k; i++) tickets[i] = sv->completed[i];
    sv->completed.erase(sv->completed.begin(), sv->completed.begin() + k);
    *n = k;
    return PB_OK;
}

int pb_serve_status(const pb_serve* sv, long long ticket, int* state, int* cycles, double* rel_res)
{
    if (!sv) return PB_ERR_ARG;
    auto it = sv->solves.find(ticket);
    if (it == sv->solves.end()) return PB_ERR_ARG;
    const SvSolve& s = it->second;
    if (state) *state = s.state;
    if (cycles) *cycles = s.cycles;
    if (rel_res) *rel_res = s.r0 > 0 ? s.r / s.r0 : 0.0;
    return PB_OK;
}

int pb_serve_timing(const pb_serve* sv, double* seconds5, long long* steps)
{
    if (!sv || !seconds5) return PB_ERR_ARG;
    for (int k = 0; k < 5; k++) seconds5[k] = sv->t_stage[k];
    if (steps) *steps = sv->steps;
    return PB_OK;
}

long long pb_serve_device_bytes(const pb_serve* sv)
{
    return sv ? (long long)sv->held : -1;
}

long long pb_serve_request_bytes(int n)
{
    return edge_ok(n) ? (long long)hier_bytes(n, false) : -1;
}

long long pb_serve_hierarchy_bytes(int n, int precision)
{
    if (precision != PB_MG_MIXED && precision != PB_MG_FP64) return -1;
    return edge_ok(n) ? (long long)hier_bytes(n, precision == PB_MG_FP64) : -1;
}

} // extern "C"
