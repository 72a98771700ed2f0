// Star-shaped stencil kernels (terms only on the axes, |offset| <= R) for sm_100a.
//
// Two kernels share the same epilogue interface:
//   k_star_tma    : TMA-staged z-streaming, warp specialised. A CTA owns a (64*XV) x TY column of
//                   output points and a chunk of z. One producer warp brings planes of the source
//                   tile (with an R-wide halo in x and y) into shared memory with
//                   cp.async.bulk.tensor, through an NST-deep ring of full/empty mbarriers; each
//                   consumer thread computes XV adjacent points in each of YB rows, keeps their z
//                   neighbours in a (2R+1)-deep register window that rotates by renaming (the z
//                   loop is unrolled by 2R+1), and reads the remaining x/y neighbours from the
//                   centre plane in shared memory.
//   k_star_simple : one thread per point, read-only cached global loads (small boxes, and any
//                   box the TMA alignment rules exclude).
//
// Terms are evaluated in the stencil's insertion order with one rounding per multiply and per add
// (no FMA), so the result is bitwise the reference's Stencil::hostApply
// (include/base/implem/Proto_StencilImplem.H:725-828 in the reference project).
#pragma once
#include <type_traits>

#include "pb_internal.cuh"

namespace pb {

// Stencil<T>::Laplacian() insertion order: 0, +x, -x, +y, -y, +z, -z (Proto_StencilDefs.H:77-87)
struct ShapeLap7 {
    static constexpr int R = 1, NT = 7, ID = 1;
    __host__ __device__ static constexpr int off(int j, int d)
    {
        return (j == 0) ? 0 : (((j - 1) / 2 == d) ? (((j - 1) % 2 == 0) ? 1 : -1) : 0);
    }
};
// sum_d Stencil<T>::Derivative(2, d, 4): per axis +e, 0, -e, +2e, -2e with the centre merged into
// the first axis' slot: +x, 0, -x, +2x, -2x, +y, -y, +2y, -2y, +z, -z, +2z, -2z
// (Proto_StencilDefs.H:393-457, composed through Stencil::operator+=)
struct ShapeLap13 {
    static constexpr int R = 2, NT = 13, ID = 2;
    __host__ __device__ static constexpr int val_x(int j) { return j == 0 ? 1 : j == 2 ? -1 : j == 3 ? 2 : j == 4 ? -2 : 0; }
    __host__ __device__ static constexpr int val_yz(int k) { return k == 0 ? 1 : k == 1 ? -1 : k == 2 ? 2 : -2; }
    __host__ __device__ static constexpr int off(int j, int d)
    {
        return (j < 5) ? (d == 0 ? val_x(j) : 0) : ((1 + (j - 5) / 4 == d) ? val_yz((j - 5) % 4) : 0);
    }
};

template <typename T>
struct Coefs {
    T c[13];
};

// Epilogues that need a second weighted sum of the same taps (a residual beside a relaxation)
// declare kTwoSums = true and provide c2 (its coefficients), init2 and finish2; the kernels then
// carry a second accumulator, summed in the same term order. Others are unaffected.
template <class E, class = void>
struct two_sums : std::false_type {};
template <class E>
struct two_sums<E, std::void_t<decltype(E::kTwoSums)>> : std::integral_constant<bool, E::kTwoSums> {};

// Geometry of one star application. Index-box point (x,y,z), 0 <= x < nx ..., maps to source-local
// coordinates (x+ox, y+oy, z+oz) in a field of extents (Sx, Sy, Sz).
struct StarGeom {
    int nx, ny, nz;
    int ox, oy, oz;
    int Sx, Sy, Sz;
    int zc;     // TMA kernel: z extent per CTA
    int pad;    // TMA kernel: shared-memory x offset of the halo start (16-byte alignment)
    int nst;    // TMA kernel: stages in the ring (>= 2R+1, <= 16)
};

constexpr int kStarTX = 64;   // consumer threads along x

template <class S, typename T, int TY, int XV>
struct StarSmem {
    static constexpr int EV = 16 / (int)sizeof(T);                  // elements per 16 bytes
    static constexpr int TXW = kStarTX * XV;                        // tile width in points
    static constexpr int BX = ((TXW + 2 * S::R + (EV - 1)) + EV - 1) / EV * EV;
    static constexpr int BY = TY + 2 * S::R;
    static constexpr int PLANE_TX = BX * BY * (int)sizeof(T);       // bytes one TMA box delivers
    static constexpr int PLANE = (PLANE_TX + 127) / 128 * 128;
};

// CTAs per SM the register budget is sized for
__host__ __device__ constexpr int star_min_blocks(int TY, int YB, int XV)
{
    return XV > 1 ? 2 : ((kStarTX * (TY / YB) + 32) <= 288 ? 3 : 2);
}

// Warp-wide max of a non-negative value followed by one atomic per warp (the warp-specialised
// kernel's consumer warps finish independently).
__device__ inline void warp_max_atomic(double v, double* result)
{
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = (v < w) ? w : v;
    }
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomic_max_nonneg(result, v);
}

// Block-wide max of a non-negative value followed by one atomic per CTA (deterministic: max is
// order independent). Every thread of the block must call it.
__device__ inline void block_max_atomic(double v, double* result)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = (v < w) ? w : v;
    }
    int nthr = blockDim.x * blockDim.y * blockDim.z;
    int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (nthr + 31) >> 5;
        double m = (lane < nw) ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            double w = __shfl_down_sync(0xffffffffu, m, o);
            m = (m < w) ? w : m;
        }
        if (lane == 0 && m > 0.0) atomic_max_nonneg(result, m);
    }
}

// Auxiliary per-point fields an epilogue reads (e.g. the right-hand side of a relaxation): up to
// three (Epi::kAux says how many the epilogue reads), each a field with its own element size and
// box. In the TMA kernel they travel through the
// same pipeline as the source planes (one tile per output plane) or are read from global memory;
// in the simple kernel they are read from global memory.
struct AuxSpec {
    const void* base;
    int esize;                 // 8 or 4 bytes
    int Sx, Sy, Sz;            // extents of the field
    int ox, oy, oz;            // field-local coordinates of index point (0,0,0)
};
constexpr int kMaxAux = 3;
struct AuxSpecs {
    int n;
    int in_smem;               // TMA kernel: 1 stages the tiles through shared memory, 0 reads global memory
    AuxSpec a[kMaxAux];
};
// What an epilogue sees: per auxiliary field, the address of this point's value.
struct AuxCtx {
    const void* p[kMaxAux];
    template <typename A>
    __device__ __forceinline__ A get(int k) const { return *reinterpret_cast<const A*>(p[k]); }
};

// shared-memory tile of one auxiliary field for one output plane: the tile's points plus room for
// the 16-byte alignment shift of the field's x origin
template <int TY, int XV>
struct AuxTile {
    static constexpr int width(int esize) { return kStarTX * XV + 16 / esize; }
    static constexpr int bytes(int esize) { return ((width(esize) * TY * esize) + 127) / 128 * 128; }
};

// Runs step(integral_constant<PH>, zo + PH) for PH = P .. W-1 while zo + PH < nzl; false when a
// step gave up (a bounded wait expired).
template <int P, int W, class F>
__device__ __forceinline__ bool run_phases(F& step, int zo, int nzl)
{
    if constexpr (P < W) {
        if (zo + P >= nzl) return true;
        if (!step(std::integral_constant<int, P>{}, zo + P)) return false;
        return run_phases<P + 1, W>(step, zo, nzl);
    } else {
        return true;
    }
}

// Warp-specialised TMA z-streaming star kernel. Threads: 64 x (TY/YB) consumers, each computing XV
// adjacent points in each of YB rows, plus one producer warp that issues the TMA copies. Stage s
// of the NST-deep ring holds source plane q (q % NST == s) and, when q - R is an output plane, the
// auxiliary tiles of that plane; full[s] completes when its bytes land, empty[s] when every
// consumer warp is done with it. Epilogues see points through a per-row cursor set up once
// (Epi::Row). Epilogues that write periodic images (Epi::kZEdge) get a separate instantiation of
// the step for the first and last plane of the domain (finish<true>), so interior planes carry no
// z-image code. Waits are bounded; on expiry the kernel flags DEV_WAIT_TIMEOUT and leaves.
template <class S, typename T, int TY, int YB, int XV, class Epi>
__global__ void __launch_bounds__(kStarTX * (TY / YB) + 32, star_min_blocks(TY, YB, XV))
    k_star_tma(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap amap0,
               const __grid_constant__ CUtensorMap amap1, const __grid_constant__ CUtensorMap amap2,
               const StarGeom g, const AuxSpecs aux, const Coefs<T> cf, const Epi epi_in)
{
    using SM = StarSmem<S, T, TY, XV>;
    using AT = AuxTile<TY, XV>;
    constexpr int R = S::R, W = 2 * R + 1;
    constexpr int NA = Epi::kAux;                     // auxiliary fields the epilogue reads
    constexpr int NCW = kStarTX * (TY / YB) / 32;     // consumer warps
    static_assert(TY % YB == 0, "rows per thread must divide the tile");
    static_assert(NA <= kMaxAux, "too many auxiliary fields");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int NST = g.nst;                            // the launcher checks 2R+1 <= NST <= 16
    const bool aux_sm = NA > 0 && aux.in_smem != 0;
    // byte offset of each auxiliary tile within a stage (aux.n <= NA fields are present)
    int aoff[kMaxAux + 1];
    aoff[0] = SM::PLANE;
#pragma unroll
    for (int k = 0; k < kMaxAux; k++)
        aoff[k + 1] = aoff[k] + ((aux_sm && k < NA && k < aux.n) ? AT::bytes(aux.a[k].esize) : 0);
    const int stage = aoff[NA];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NST * stage);
    uint64_t* empty = full + NST;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * SM::TXW, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * g.zc;
    const int nzl = min(g.zc, g.nz - zb);
    if (nzl <= 0) return;
    const int nplanes = nzl + 2 * R;

    if (tid == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp == NCW) {
        // ---- producer warp ----
        if (lane == 0) {
            const int xs = g.ox + x0 - R - g.pad, ys = g.oy + y0 - R, zs0 = g.oz + zb - R;
            int s = 0;
            uint32_t eph = 0;   // parity bits of the next empty-wait per slot
            int issued = 0;
            for (int q = 0; q < nplanes; q++) {
                if (q >= NST) {
                    if (!mbar_wait(&empty[s], (eph >> s) & 1)) break;
                    eph ^= 1u << s;
                }
                unsigned char* st = smem_raw + s * stage;
                const int zo = q - R;
                const bool with_aux = aux_sm && zo >= 0 && zo < nzl;
                uint32_t bytes = SM::PLANE_TX;
                if (with_aux) {
#pragma unroll
                    for (int k = 0; k < NA; k++)
                        if (k < aux.n) bytes += AT::width(aux.a[k].esize) * TY * aux.a[k].esize;
                }
                mbar_arrive_expect_tx(&full[s], bytes);
                tma_load_3d(st, &tmap, &full[s], xs, ys, zs0 + q);
                if (with_aux) {
#pragma unroll
                    for (int k = 0; k < NA; k++) {
                        if (k >= aux.n) break;
                        const AuxSpec& a = aux.a[k];
                        const CUtensorMap* am = k == 0 ? &amap0 : (k == 1 ? &amap1 : &amap2);
                        tma_load_3d(st + aoff[k], am, &full[s], a.ox + x0 - (a.ox % (16 / a.esize)), a.oy + y0,
                                    a.oz + zb + zo);
                    }
                }
                if (++s == NST) s = 0;
                issued = q + 1;
            }
            // Copies still in flight must land before the CTA's shared memory goes away (the consumers
            // wait for every plane on a normal exit; this covers an exit after a timed-out wait).
            for (int q = max(0, issued - NST); q < issued; q++) mbar_wait(&full[q % NST], (q / NST) & 1);
        }
        return;
    }

    // ---- consumer warps ----
    Epi epi = epi_in;
    const int tx = tid & (kStarTX - 1), ty = tid / kStarTX;
    const int x = x0 + tx * XV;                            // first of this thread's XV points
    const int yr0 = ty * YB;                               // first tile row of this thread
    const bool xin = x < g.nx;                             // XV > 1: the launcher ensures nx % XV == 0
    const int sc0 = (yr0 + R) * SM::BX + (tx * XV + R + g.pad);   // centre element of the first point
    typename Epi::Row rows[YB];
#pragma unroll
    for (int r = 0; r < YB; r++) {
        const int y = y0 + yr0 + r;
        rows[r] = epi.row(x, y, zb, xin && (y < g.ny));
    }
    // auxiliary-field address of row r, point v: base + abase + r * arow + v * esize
    long long abase[kMaxAux], astep[kMaxAux];
    int arow[kMaxAux], es[kMaxAux];
#pragma unroll
    for (int k = 0; k < NA; k++) {
        const AuxSpec& a = aux.a[k];
        es[k] = a.esize;
        astep[k] = 0;
        if (aux_sm) {
            const int w = AT::width(a.esize);
            abase[k] = ((long long)yr0 * w + tx * XV + a.ox % (16 / a.esize)) * a.esize;
            arow[k] = w * a.esize;
        } else {
            const int y = y0 + yr0;
            abase[k] = ((x + a.ox) + (long long)a.Sx * ((y + a.oy) + (long long)a.Sy * (zb + a.oz))) * a.esize;
            arow[k] = a.Sx * a.esize;
            astep[k] = (long long)a.Sx * a.Sy * a.esize;
        }
    }
    T win[YB][XV][W];
    bool ok = true;
    // window: planes 0 .. 2R-1 (slots 0 .. 2R-1 of the ring, first use: parity 0)
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        ok &= mbar_wait(&full[q], 0);
        const T* pl = reinterpret_cast<const T*>(smem_raw + q * stage);
#pragma unroll
        for (int r = 0; r < YB; r++)
#pragma unroll
            for (int v = 0; v < XV; v++) win[r][v][q] = pl[sc0 + r * SM::BX + v];
    }
    __syncwarp();
    // planes 0 .. R-1 only fed the window
    if (lane == 0)
        for (int q = 0; q < R; q++) mbar_arrive(&empty[q]);
    ok = __all_sync(0xffffffffu, ok);
    int sn = 2 * R;        // slot of the newest plane (NST > 2R)
    uint32_t pn = 0;       // its phase parity
    int scs = R;           // slot of the centre plane

    // One z step. PH = zo mod (2R+1) names the window slots, so the window rotates by renaming;
    // ZE: this plane is the first or last of the domain (periodic z images).
    auto step_ze = [&](auto PHc, auto ZEc, int zo) -> bool {
        constexpr int PH = decltype(PHc)::value;
        constexpr bool ZE = decltype(ZEc)::value;
        constexpr int IN = (PH + 2 * R) % W, IC = (PH + R) % W;
        if (!__all_sync(0xffffffffu, mbar_wait(&full[sn], pn))) return false;
        const T* pnew = reinterpret_cast<const T*>(smem_raw + sn * stage);
#pragma unroll
        for (int r = 0; r < YB; r++)
#pragma unroll
            for (int v = 0; v < XV; v++) win[r][v][IN] = pnew[sc0 + r * SM::BX + v];
        const unsigned char* stc = smem_raw + scs * stage;
        const T* pc = reinterpret_cast<const T*>(stc);
        const unsigned char* ab[kMaxAux];
#pragma unroll
        for (int k = 0; k < NA; k++)
            ab[k] = (aux_sm ? stc + aoff[k] : reinterpret_cast<const unsigned char*>(aux.a[k].base) + zo * astep[k]) +
                    abase[k];
#pragma unroll
        for (int r = 0; r < YB; r++) {
#pragma unroll
            for (int v = 0; v < XV; v++) {
                AuxCtx ax;
#pragma unroll
                for (int k = 0; k < NA; k++) ax.p[k] = ab[k] + r * arow[k] + v * es[k];
                T acc = epi.init(rows[r], zo, v, ax);
                [[maybe_unused]] T acc2 = T(0);
                if constexpr (two_sums<Epi>::value) acc2 = epi.init2(rows[r], zo, v, ax);
#pragma unroll
                for (int j = 0; j < S::NT; j++) {
                    const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
                    T val;
                    if (oz != 0) val = win[r][v][(IC + oz + W) % W];
                    else if (ox == 0 && oy == 0) val = win[r][v][IC];
                    else if (oy == 0 && v + ox >= 0 && v + ox < XV) val = win[r][v + ox][IC];   // this thread's point
                    else if (ox == 0 && r + oy >= 0 && r + oy < YB) val = win[r + oy][v][IC];   // this thread's row
                    else val = pc[sc0 + (r + oy) * SM::BX + v + ox];
                    acc = dmadd(acc, cf.c[j], val);
                    if constexpr (two_sums<Epi>::value) acc2 = dmadd(acc2, epi.c2.c[j], val);
                }
                if constexpr (two_sums<Epi>::value) epi.template finish2<ZE>(rows[r], zo, v, acc, acc2, win[r][v][IC], ax);
                else epi.template finish<ZE>(rows[r], zo, v, acc, win[r][v][IC], ax);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[scs]);
        if (++sn == NST) {
            sn = 0;
            pn ^= 1;
        }
        if (++scs == NST) scs = 0;
        return true;
    };
    auto step = [&](auto PHc, int zo) -> bool {
        if constexpr (Epi::kZEdge) {
            if (epi.z_edge(zb + zo)) return step_ze(PHc, std::true_type{}, zo);
        }
        return step_ze(PHc, std::false_type{}, zo);
    };
    if (ok) {
        for (int zo = 0; zo < nzl; zo += W)
            if (!run_phases<0, W>(step, zo, nzl)) break;
    }
    epi.end_warp();
}

// One thread per point (small boxes and any box the TMA rules exclude).
template <class S, typename T, class Epi>
__global__ void __launch_bounds__(256) k_star_simple(const T* __restrict__ src, const StarGeom g, const AuxSpecs aux,
                                                     const Coefs<T> cf, const Epi epi_in)
{
    Epi epi = epi_in;
    const long long total = (long long)g.nx * g.ny * g.nz;
    const long long Sx = g.Sx, Sxy = (long long)g.Sx * g.Sy;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % g.nx);
        long long r = i / g.nx;
        int y = (int)(r % g.ny);
        int z = (int)(r / g.ny);
        long long base = (x + g.ox) + Sx * (y + g.oy) + Sxy * (z + g.oz);
        AuxCtx ax;
#pragma unroll
        for (int k = 0; k < Epi::kAux; k++) {
            const AuxSpec& a = aux.a[k];
            ax.p[k] = reinterpret_cast<const unsigned char*>(a.base) +
                      ((x + a.ox) + (long long)a.Sx * ((y + a.oy) + (long long)a.Sy * (z + a.oz))) * a.esize;
        }
        const typename Epi::Row row = epi.row(x, y, z, true);
        T acc = epi.init(row, 0, 0, ax);
        [[maybe_unused]] T acc2 = T(0);
        if constexpr (two_sums<Epi>::value) acc2 = epi.init2(row, 0, 0, ax);
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const long long o = S::off(j, 0) + Sx * S::off(j, 1) + Sxy * S::off(j, 2);
            const T val = __ldg(src + base + o);
            acc = dmadd(acc, cf.c[j], val);
            if constexpr (two_sums<Epi>::value) acc2 = dmadd(acc2, epi.c2.c[j], val);
        }
        bool ze = false;
        if constexpr (Epi::kZEdge) ze = epi.z_edge(z);
        if constexpr (two_sums<Epi>::value) {
            if (ze) epi.template finish2<true>(row, 0, 0, acc, acc2, __ldg(src + base), ax);
            else epi.template finish2<false>(row, 0, 0, acc, acc2, __ldg(src + base), ax);
        } else {
            if (ze) epi.template finish<true>(row, 0, 0, acc, __ldg(src + base), ax);
            else epi.template finish<false>(row, 0, 0, acc, __ldg(src + base), ax);
        }
    }
    epi.end_block();
}

// ---- basic epilogues ---------------------------------------------------------------------------
// Epilogue interface (both kernels):
//   Row                      per-row cursor type
//   kZEdge                   whether some planes need separate handling (then z_edge(z) says which)
//   kAux                     how many auxiliary fields init/finish read (AuxCtx::get<A>(k), k < kAux)
//   row(x, y, z0, active)    cursor of the row of points x .. x+XV-1 at y, starting at plane z0
//   init(row, zo, v, ax)     accumulator start for point v of the row at plane z0+zo
//   finish<ZE>(row, zo, v, acc, c, ax)   consume the stencil sum (c = the source's centre value)
//   end_warp() / end_block() after the TMA / simple kernel's last point
// Output addressing for a field on a box: index-box point (x,y,z) -> (x+dx) + Dx*(y+dy) + Dxy*(z+dz)
struct OutMap {
    long long dx, dy, dz, Dx, Dxy;
    __device__ __forceinline__ long long at(int x, int y, int z) const { return (x + dx) + Dx * (y + dy) + Dxy * (z + dz); }
};

// Per-row output cursor: the row's address at its first z and whether the row is inside the box.
template <typename T>
struct OutRow {
    T* p;
    bool active;
};

// "dst |= S(src)" (init 0) and "dst += S(src)" (init = old dst value, then the terms)
template <typename T>
struct EpiStore {
    T* dst;
    OutMap m;
    int accumulate;
    using Row = OutRow<T>;
    static constexpr bool kZEdge = false;
    static constexpr int kAux = 0;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const { return Row{dst + m.at(x, y, z0), active}; }
    __device__ __forceinline__ T init(const Row& r, int zo, int v, const AuxCtx&) const
    {
        return (accumulate && r.active) ? r.p[zo * m.Dxy + v] : T(0);
    }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int v, T acc, T, const AuxCtx&) const
    {
        if (r.active) r.p[zo * m.Dxy + v] = acc;
    }
    __device__ __forceinline__ bool z_edge(int) const { return false; }
    __device__ __forceinline__ void end_warp() const {}
    __device__ __forceinline__ void end_block() const {}
};

// out = a*Lu + b*u  /  out = u + a*Lu
template <typename T>
struct EpiAxpby {
    T* dst;
    OutMap m;
    T a, b;
    int euler;
    using Row = OutRow<T>;
    static constexpr bool kZEdge = false;
    static constexpr int kAux = 0;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const { return Row{dst + m.at(x, y, z0), active}; }
    __device__ __forceinline__ T init(const Row&, int, int, const AuxCtx&) const { return T(0); }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int v, T acc, T u, const AuxCtx&) const
    {
        if (r.active) r.p[zo * m.Dxy + v] = euler ? dadd(u, dmul(a, acc)) : dadd(dmul(a, acc), dmul(b, u));
    }
    __device__ __forceinline__ bool z_edge(int) const { return false; }
    __device__ __forceinline__ void end_warp() const {}
    __device__ __forceinline__ void end_block() const {}
};

} // namespace pb
