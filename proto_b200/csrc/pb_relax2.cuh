// Two weighted-Jacobi sweeps of a periodic multigrid level in one pass over HBM (temporal blocking).
//
// phi2 = relax(relax(phi0)): the level is read once (phi0, rho, alpha) and written once (phi2 with
// its periodic ghost images) instead of twice each, so the pair moves 24 (FP64) / 12 (FP32) bytes
// per cell where two separate sweeps move 48 / 24. The intermediate phi1 never leaves the SM.
//
// A CTA owns TY = 2*RG full-length rows (all n cells of x) of a chunk of zc planes and streams in z.
// Full rows make the x direction periodic by index arithmetic alone (the grown row carries the
// ghost columns of phi0; phi1's x neighbours wrap modulo n in shared memory), so only y and z need
// explicit wrapping, which the producer does by choosing the rows and planes it copies.
//   producer warp : copies, per plane, the phi0 tile (TY + 4 rows: the tile, one ring row of phi1
//                   on each side and one more for phi1's own y taps) and the rho (and alpha) tile of
//                   the TY + 2 phi1 rows into an NST-deep shared-memory ring with
//                   cp.async.bulk.tensor (one box per x segment of the whole tile, one per row where
//                   the tile wraps in y); full/empty mbarriers.
//   stencil warps : two groups of NXT threads; group 0 owns output rows y0 .. y0+RG-1 plus the ring
//                   row y0-1, group 1 rows y0+RG .. y0+TY-1 plus the ring row y0+TY. Lane l of warp
//                   w of a group takes the PV cells x = 32*PV*w + 32*v + l (v < PV) of each of its
//                   rows (consecutive lanes on consecutive cells: conflict-free shared memory,
//                   coalesced global stores). Per plane p, a group computes phi1(p) on its RG + 1
//                   rows (z taps from a three-plane register window of phi0, x/y taps from the
//                   centre plane in shared memory), publishes them to a double-buffered phi1 plane
//                   in shared memory, and computes phi2(p-1) on its RG output rows (z taps from a
//                   register window of its own phi1 rows, x/y taps at its edges from the published
//                   plane). One named barrier per plane orders the phi1 planes between the groups;
//                   a stage returns to the producer as soon as phi1 of its plane is computed (the
//                   right-hand side phi2 needs a plane later stays in registers).
// Every phi1 and phi2 value is computed with EpiRelax's arithmetic (taps in the 7-point
// Laplacian's insertion order, one rounding per operation, relax_value), from the same inputs, so
// the result is bitwise two launches of the single-sweep kernel. With NORM the pass also takes the
// max-norm residual of phi0 (EpiRelaxNorm's second sum) at the cells of its own rows and planes,
// so at every cell of the level once.
// Modes: kRelax2Plain; kRelax2Zero, the pair that starts a level from zero (phi1 = the sweep of a
// zero state, from rho and alpha alone, as the first-sweep kernel computes it: no phi0 is read);
// kRelax2Update (FP32, mixed precision), the pair that ends a cycle: phi2 is not stored but added
// to the FP64 solution (u += (double)phi2, with u's periodic images), as the fused last-sweep
// update computes it.
// Waits are bounded: a stencil thread whose wait expires makes every stencil thread leave at the
// next barrier (barrier reduction), and the producer drains its copies in flight before the CTA
// exits.
#pragma once
#include "pb_mg_kernels.cuh"

namespace pb {

enum Relax2Mode : int { kRelax2Plain = 0, kRelax2Zero = 1, kRelax2Update = 2 };

template <typename T>
struct Relax2Args {
    T* out;                 // destination level (grown, pitch k.sx)
    double* u;              // kRelax2Update: FP64 solution (grown, pitch usx)
    int usx;
    RelaxCoef<T> k;         // n, sx, form and the smoother's scalars
    Coefs<T> c;             // smoother taps: L(., omega/6) (Poisson) | L(., 1/h^2) (Helmholtz)
    Coefs<T> c2;            // NORM: L(., 1/h^2)
    T beta;                 // NORM, Helmholtz
    double* result;         // NORM: max-norm accumulator (atomic max)
    int zc;                 // planes per CTA
    int nst;                // ring stages (3 .. 6)
    int nb, bw;             // x segments per copied phi0 row and their width in elements
};

// Named barrier of the stencil threads with an OR over a predicate (bar.red): every one gets the
// same answer, so a bounded wait that expired anywhere ends the loop everywhere at once.
__device__ __forceinline__ bool consumers_any(bool pred, int nthreads)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(nthreads)
        : "memory");
    return r != 0;
}

// grown index (ghost layer included) of logical coordinate c in [-2, n+1] of a periodic n-cell axis:
// -1 and n are the ghost layer; -2 and n+1 wrap to the valid cells n-2 and 1
__host__ __device__ __forceinline__ int r2_grown(int c, int n)
{
    return c < -1 ? c + n + 1 : (c > n ? c - n + 1 : c + 1);
}
// logical coordinate c in [-2, n+1] of a periodic n-cell axis wrapped into [0, n)
__device__ __forceinline__ int r2_wrap(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// NXT threads per group, each taking PV cells of a row, so the level edge is N = NXT * PV.
template <int NXT, int PV, int RG>
struct Relax2Shape {
    static constexpr int N = NXT * PV;             // level edge
    static constexpr int TY = 2 * RG;              // output rows per CTA
    static constexpr int ROWS = TY + 4;            // phi0 rows copied per plane
    static constexpr int B1ROWS = TY + 2;          // phi1 rows per plane (and rho rows copied)
    static constexpr int NC = 2 * NXT;             // stencil threads
    static constexpr int NCW = NC / 32;            // their warps
    static constexpr int THREADS = NC + 32;        // and the producer warp
};

__host__ __device__ constexpr int relax2_min_blocks(int threads)
{
    return threads <= 160 ? 3 : (threads <= 288 ? 2 : 1);
}

template <typename T, int NXT, int PV, int RG, bool HELM, bool NORM, int MODE>
__global__ void __launch_bounds__(2 * NXT + 32, relax2_min_blocks(2 * NXT + 32))
    k_relax2(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmapE,
             const __grid_constant__ CUtensorMap tmap1, const __grid_constant__ CUtensorMap rmap,
             const __grid_constant__ CUtensorMap rmapE, const __grid_constant__ CUtensorMap rmap1,
             const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap amapE,
             const __grid_constant__ CUtensorMap amap1, const Relax2Args<T> a)
{
    using SH = Relax2Shape<NXT, PV, RG>;
    constexpr int N = SH::N, TY = SH::TY, J = RG + 1, NA = HELM ? 2 : 1;
    constexpr bool ZERO = MODE == kRelax2Zero, UPD = MODE == kRelax2Update;
    static_assert(NXT % 32 == 0, "groups are whole warps");
    static_assert(!(NORM && MODE != kRelax2Plain), "the norm rides on plain passes only");
    static_assert(!UPD || sizeof(T) == 4, "the update pass belongs to mixed precision");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nst = a.nst;
    const int tile0 = ZERO ? 0 : SH::ROWS * a.nb * a.bw;        // phi0 tile (elements; none from zero)
    const int tilea = SH::B1ROWS * N;                           // rho / alpha tile (elements)
    const int stage_bytes = (tile0 + NA * tilea) * (int)sizeof(T);   // multiple of 128
    T* b1 = reinterpret_cast<T*>(smem_raw + nst * stage_bytes); // phi1 planes [2][B1ROWS][N]
    uint64_t* full = reinterpret_cast<uint64_t*>(b1 + 2 * tilea);
    uint64_t* empty = full + nst;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = blockIdx.x * TY;
    const int zb = blockIdx.y * a.zc;
    const int nzl = min(a.zc, N - zb);
    const int nplanes = nzl + 4;                                // planes zb-2 .. zb+nzl+1

    if (tid == 0) {
        for (int s = 0; s < nst; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], SH::NCW);
        }
        fence_barrier_init();
    }
    __syncthreads();

    constexpr int NBR = N > 256 ? 2 : 1, BWR = N / NBR;         // rho / alpha segments per row
    if (warp == SH::NCW) {
        // ---- producer: plane kp (= zb-2+kp, wrapped) into stage kp % nst: the phi0 tile (rows
        // y0-2 .. y0+TY+1) and the rho (and alpha) tile (rows y0-1 .. y0+TY). Inside the domain the
        // rows of a tile are contiguous, so each x segment is one box of all its rows. The first
        // and last row tiles wrap in y by one row: each segment is one box of the other rows (one
        // row shorter) and one single-row box of the wrapped row. Shared memory holds each segment
        // as a dense [rows][width] block either way. ----
        if (lane == 0) {
            const bool inner = y0 >= 1 && y0 + TY <= N - 1;
            const bool top = y0 == 0;                    // else the last tile (y0 + TY == N)
            const int row_bytes0 = a.bw * (int)sizeof(T), row_bytesr = BWR * (int)sizeof(T);
            // first tile: wrapped row first, then the rest from grown row 0 (phi0) / row 0 (rho);
            // last tile: the rest from grown row N-TY-1 / row N-TY-1, then the wrapped row
            const int e0_dst = top ? 1 : 0, e0_y = top ? 0 : N - TY - 1, w0_dst = top ? 0 : SH::ROWS - 1,
                      w0_y = top ? N - 1 : 2;
            const int er_dst = top ? 1 : 0, er_y = top ? 0 : N - TY - 1, wr_dst = top ? 0 : SH::B1ROWS - 1,
                      wr_y = top ? N - 1 : 0;
            int issued = 0;
            for (int kp = 0; kp < nplanes; kp++) {
                const int s = kp % nst;
                if (kp >= nst && !mbar_wait(&empty[s], ((kp / nst) - 1) & 1)) break;
                const int q = zb - 2 + kp;
                const int gz = r2_grown(q, N), wz = r2_wrap(q, N);
                unsigned char* st = smem_raw + s * stage_bytes;
                unsigned char* sr = st + tile0 * (int)sizeof(T);
                mbar_arrive_expect_tx(&full[s], (uint32_t)stage_bytes);
                if (inner) {
                    if constexpr (MODE != kRelax2Zero) {
                        for (int xb = 0; xb < a.nb; xb++)
                            tma_load_3d(st + xb * SH::ROWS * a.bw * (int)sizeof(T), &tmap, &full[s], xb * a.bw, y0 - 1,
                                        gz);
                    }
#pragma unroll
                    for (int xb = 0; xb < NBR; xb++) {
                        unsigned char* d = sr + xb * SH::B1ROWS * BWR * (int)sizeof(T);
                        tma_load_3d(d, &rmap, &full[s], xb * BWR, y0 - 1, wz);
                        if constexpr (HELM) tma_load_3d(d + tilea * (int)sizeof(T), &amap, &full[s], xb * BWR, y0 - 1, wz);
                    }
                } else {
                    if constexpr (MODE != kRelax2Zero) {
                        for (int xb = 0; xb < a.nb; xb++) {
                            unsigned char* d = st + xb * SH::ROWS * row_bytes0;
                            tma_load_3d(d + e0_dst * row_bytes0, &tmapE, &full[s], xb * a.bw, e0_y, gz);
                            tma_load_3d(d + w0_dst * row_bytes0, &tmap1, &full[s], xb * a.bw, w0_y, gz);
                        }
                    }
#pragma unroll
                    for (int xb = 0; xb < NBR; xb++) {
                        unsigned char* d = sr + xb * SH::B1ROWS * row_bytesr;
                        tma_load_3d(d + er_dst * row_bytesr, &rmapE, &full[s], xb * BWR, er_y, wz);
                        tma_load_3d(d + wr_dst * row_bytesr, &rmap1, &full[s], xb * BWR, wr_y, wz);
                        if constexpr (HELM) {
                            unsigned char* da = d + tilea * (int)sizeof(T);
                            tma_load_3d(da + er_dst * row_bytesr, &amapE, &full[s], xb * BWR, er_y, wz);
                            tma_load_3d(da + wr_dst * row_bytesr, &amap1, &full[s], xb * BWR, wr_y, wz);
                        }
                    }
                }
                issued = kp + 1;
            }
            // copies in flight land before the CTA's shared memory goes away
            for (int kp = max(0, issued - nst); kp < issued; kp++) mbar_wait(&full[kp % nst], (kp / nst) & 1);
        }
        return;
    }

    // ---- stencil work ----
    const int g = tid / NXT;                  // warp-uniform (NXT is a multiple of 32)
    const int tg = tid - g * NXT;             // thread within the group
    int xs[PV];
#pragma unroll
    for (int v = 0; v < PV; v++) xs[v] = (tg >> 5) * 32 * PV + 32 * v + lane;
    // tile element of (row ly, grown x gx) = col0(gx) + ly * bw (phi0: segment-major blocks); of
    // (row r, x) in the rho tile = colr(x) + r * BWR
    const int bw = a.bw;
    auto col0 = [&](int gx) { return (gx / bw) * SH::ROWS * bw + gx % bw; };
    int cm[PV], cc[PV], cp[PV], cr[PV];
#pragma unroll
    for (int v = 0; v < PV; v++) {
        cm[v] = col0(xs[v]);
        cc[v] = col0(xs[v] + 1);
        cp[v] = col0(xs[v] + 2);
        cr[v] = (xs[v] / BWR) * SH::B1ROWS * BWR + xs[v] % BWR;
    }

    const RelaxCoef<T> k = a.k;
    const int sx = k.sx;
    const long long Sz = (long long)sx * (N + 2);

    auto run = [&](auto Gc) {
        constexpr int G = decltype(Gc)::value;
        constexpr int JO = G == 0 ? 1 : 0;           // phi1 row of output row r: j = r + JO
        const int ys = y0 - 1 + G * (RG + 1);         // logical y of phi1 row j = ys + j
        const int ly0 = G * (RG + 1) + 1;             // phi0 tile row of phi1 row 0
        const int br0 = G * (RG + 1);                 // phi1 plane / rho tile row of phi1 row 0
        // output cursor: valid cell (xs[0], y of output row 0, plane) of the destination, advanced one
        // plane per phi2 plane; row r, cell v at + r * sx + 32 * v. Periodic image offsets per cell
        // in x and per row in y, and the phi1 plane's x neighbours (wrapped), fixed per thread.
        T* orow = a.out + grown_index<T>(N, sx, xs[0], ys + JO, zb);
        // kRelax2Update: the FP64 solution's cursor, pitch usx, images per row in y
        [[maybe_unused]] double* urow = nullptr;
        [[maybe_unused]] int uyr[MODE == kRelax2Update ? RG : 1] = {};
        [[maybe_unused]] long long Suz = 0;
        if constexpr (MODE == kRelax2Update) {
            urow = a.u + grown_index<double>(N, a.usx, xs[0], ys + JO, zb);
            Suz = (long long)a.usx * (N + 2);
#pragma unroll
            for (int r = 0; r < RG; r++) uyr[r] = image_offset(ys + JO + r, N, a.usx);
        }
        int oxv[PV], xmv[PV], xpv[PV], oyr[RG];
#pragma unroll
        for (int v = 0; v < PV; v++) {
            oxv[v] = image_offset(xs[v], N, 1);
            xmv[v] = xs[v] == 0 ? N - 1 : xs[v] - 1;
            xpv[v] = xs[v] == N - 1 ? 0 : xs[v] + 1;
        }
#pragma unroll
        for (int r = 0; r < RG; r++) oyr[r] = image_offset(ys + JO + r, N, sx);
        // relax_value with the form fixed at compile time (the same operations in the same order)
        auto rv = [&](T acc, T c, T rho, T al) -> T {
            if constexpr (!HELM) return dadd(c, dmadd(acc, k.neg_lambda, rho));
            else {
                const T r = dsub(rho, dsub(dmul(al, c), dmul(k.beta, acc)));
                return dadd(c, squot(dmul(k.omega, r), dadd(al, k.diagB)));
            }
        };

        T w0[3][J][PV];            // phi0 window: [plane slot][phi1 row][cell]
        T p1[3][RG][PV];           // phi1 of the output rows: [plane slot][row][cell]
        T ro2[RG][PV];             // rho of the output rows at the plane of the last phi1 (for phi2)
        [[maybe_unused]] T ao2[HELM ? RG : 1][PV];
        [[maybe_unused]] double m = 0.0;

        // ring slots of the planes in use, advanced by one per step (no division in the loop):
        // sc = slot of the centre plane (kp t+1), sn = the new one (t+2), pn the parity of sn's fill
        int sc = 1, sn = 2;
        uint32_t pn = 0;
        auto stage = [&](int slot) -> const T* { return reinterpret_cast<const T*>(smem_raw + slot * stage_bytes); };
        auto load_window = [&](auto SLc, int slot) {
            constexpr int SL = decltype(SLc)::value;
            const T* t = stage(slot) + ly0 * bw;
#pragma unroll
            for (int j = 0; j < J; j++)
#pragma unroll
                for (int v = 0; v < PV; v++) w0[SL][j][v] = t[j * bw + cc[v]];
        };

        // prologue: phi0 planes zb-2 (kp 0) and zb-1 (kp 1) into window slots 0 and 1
        const bool ok = mbar_wait(&full[0], 0) && mbar_wait(&full[1], 0);
        if (ok && !ZERO) {
            load_window(std::integral_constant<int, 0>{}, 0);
            load_window(std::integral_constant<int, 1>{}, 1);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[0]);    // plane zb-2 only feeds the window

        // Step t: phi1 at plane p = zb-1+t from the window (planes p-1, p, p+1) and stage t+1 (the
        // centre plane's x/y taps and rho(p)), which is released at once; then phi2 at plane p-1
        // (rho(p-1) of the output rows kept in registers since the last step).
        auto step = [&](auto PHc, int t) -> bool {
            constexpr int PH = decltype(PHc)::value;          // t % 3
            constexpr int SO = PH, SC = (PH + 1) % 3, SN = (PH + 2) % 3;
            const int p = zb - 1 + t;
            const bool got = mbar_wait(&full[sn], pn);
            if (got && !ZERO) load_window(std::integral_constant<int, SN>{}, sn);
            if (consumers_any(!got, SH::NC)) return false;
            // kRelax2Update: the FP64 solution under this step's phi2 outputs (plane p-1), read now so
            // the loads overlap phi1
            [[maybe_unused]] double uin[MODE == kRelax2Update ? RG : 1][PV];
            if constexpr (MODE == kRelax2Update) {
                if (t >= 2) {
#pragma unroll
                    for (int r = 0; r < RG; r++)
#pragma unroll
                        for (int v = 0; v < PV; v++) uin[r][v] = urow[r * a.usx + 32 * v];
                }
            }
            // ---- phi1(p) on rows j ----
            T rn[RG][PV];
            [[maybe_unused]] T an[HELM ? RG : 1][PV];
            const T* cst = stage(sc);
            const T* c = cst + ly0 * bw;
            const T* rt = cst + tile0 + br0 * BWR;            // rho(p) of phi1 row 0
            T* b1w = b1 + (t & 1) * tilea + br0 * N;
            // all rows are computed before any is published: a store between them would keep the
            // next row's shared-memory loads behind it (the compiler cannot tell the buffers apart),
            // serialising the rows' independent chains
            T v1s[J][PV];
            [[maybe_unused]] const bool own_plane = t >= 1 && t <= nzl;   // p in [zb, zb + nzl)
#pragma unroll
            for (int j = 0; j < J; j++) {
#pragma unroll
                for (int v = 0; v < PV; v++) {
                    const T rho = rt[j * BWR + cr[v]];
                    T al = T(0);
                    if constexpr (HELM) al = rt[tilea + j * BWR + cr[v]];
                    T v1, tc = T(0), tpx = T(0), tmx = T(0), tpy = T(0), tmy = T(0), tpz = T(0), tmz = T(0);
                    if constexpr (MODE == kRelax2Zero) {
                        v1 = rv(T(0), T(0), rho, al);      // the sweep of a zero state
                    } else {
                        const T* q = c + j * bw;
                        tc = w0[SC][j][v];
                        tpx = q[cp[v]];
                        tmx = q[cm[v]];
                        tpy = j + 1 < J ? w0[SC][j + 1][v] : q[bw + cc[v]];
                        tmy = j > 0 ? w0[SC][j - 1][v] : q[cc[v] - bw];
                        tpz = w0[SN][j][v];
                        tmz = w0[SO][j][v];
                        T acc = T(0);
                        acc = dmadd(acc, a.c.c[0], tc);
                        acc = dmadd(acc, a.c.c[1], tpx);
                        acc = dmadd(acc, a.c.c[2], tmx);
                        acc = dmadd(acc, a.c.c[3], tpy);
                        acc = dmadd(acc, a.c.c[4], tmy);
                        acc = dmadd(acc, a.c.c[5], tpz);
                        acc = dmadd(acc, a.c.c[6], tmz);
                        v1 = rv(acc, tc, rho, al);
                    }
                    // the norm at the tile's own rows and planes only: every cell of the level once
                    if (NORM && j - JO >= 0 && j - JO < RG && own_plane) {
                        T a2 = HELM ? T(0) : dsub(T(0), rho);
                        a2 = dmadd(a2, a.c2.c[0], tc);
                        a2 = dmadd(a2, a.c2.c[1], tpx);
                        a2 = dmadd(a2, a.c2.c[2], tmx);
                        a2 = dmadd(a2, a.c2.c[3], tpy);
                        a2 = dmadd(a2, a.c2.c[4], tmy);
                        a2 = dmadd(a2, a.c2.c[5], tpz);
                        a2 = dmadd(a2, a.c2.c[6], tmz);
                        if constexpr (!HELM) m = upd_abs(m, (double)a2);
                        else m = upd_abs(m, (double)dsub(rho, dsub(dmul(al, tc), dmul(a.beta, a2))));
                    }
                    v1s[j][v] = v1;
                    const int r = j - JO;   // output row of phi1 row j (a constant once unrolled)
                    if (r >= 0 && r < RG) p1[PH][r < 0 ? 0 : (r >= RG ? RG - 1 : r)][v] = v1;
                    if (r >= 0 && r < RG) {
                        rn[r < 0 ? 0 : (r >= RG ? RG - 1 : r)][v] = rho;
                        if constexpr (HELM) an[r < 0 ? 0 : (r >= RG ? RG - 1 : r)][v] = al;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < J; j++)
#pragma unroll
                for (int v = 0; v < PV; v++) b1w[j * N + xs[v]] = v1s[j][v];
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[sc]);   // centre plane done (its taps and rho)
            // ---- phi2(p-1) on the output rows ----
            if (t >= 2) {
                constexpr int QC = (PH + 2) % 3, QP = PH, QM = (PH + 1) % 3;   // phi1 planes p-1, p, p-2
                const T* b1r = b1 + ((t - 1) & 1) * tilea + (br0 + JO) * N;   // output row 0
                const int ez = edge_code(p - 1, N);
                const long long ozv = ez == 1 ? (long long)N * Sz : -(long long)N * Sz;
                T v2s[RG][PV];
#pragma unroll
                for (int r = 0; r < RG; r++) {
#pragma unroll
                    for (int v = 0; v < PV; v++) {
                        const int x = xs[v];
                        const T tc = p1[QC][r][v];
                        const T tpx = b1r[r * N + xpv[v]], tmx = b1r[r * N + xmv[v]];
                        const T tpy = r + 1 < RG ? p1[QC][r + 1][v] : b1r[(r + 1) * N + x];
                        const T tmy = r > 0 ? p1[QC][r - 1][v] : b1r[(r - 1) * N + x];
                        const T tpz = p1[QP][r][v], tmz = p1[QM][r][v];
                        T acc = T(0);
                        acc = dmadd(acc, a.c.c[0], tc);
                        acc = dmadd(acc, a.c.c[1], tpx);
                        acc = dmadd(acc, a.c.c[2], tmx);
                        acc = dmadd(acc, a.c.c[3], tpy);
                        acc = dmadd(acc, a.c.c[4], tmy);
                        acc = dmadd(acc, a.c.c[5], tpz);
                        acc = dmadd(acc, a.c.c[6], tmz);
                        T al = T(0);
                        if constexpr (HELM) al = ao2[r][v];
                        v2s[r][v] = rv(acc, tc, ro2[r][v], al);
                    }
                }
                // stores after every row's value (global stores would otherwise order the next
                // row's shared-memory loads behind them)
                if constexpr (MODE == kRelax2Update) {
                    const long long ouz = ez == 1 ? (long long)N * Suz : -(long long)N * Suz;
#pragma unroll
                    for (int r = 0; r < RG; r++) {
#pragma unroll
                        for (int v = 0; v < PV; v++) {
                            const double v2 = dadd(uin[r][v], (double)v2s[r][v]);
                            double* q = urow + r * a.usx + 32 * v;
                            const int ox = oxv[v], oy = uyr[r];
                            *q = v2;
                            if (ox) q[ox] = v2;
                            if (oy) {
                                q[oy] = v2;
                                if (ox) q[oy + ox] = v2;
                            }
                            if (ez) {
                                double* qz = q + ouz;
                                *qz = v2;
                                if (ox) qz[ox] = v2;
                                if (oy) {
                                    qz[oy] = v2;
                                    if (ox) qz[oy + ox] = v2;
                                }
                            }
                        }
                    }
                    urow += Suz;
                } else {
#pragma unroll
                for (int r = 0; r < RG; r++) {
#pragma unroll
                    for (int v = 0; v < PV; v++) {
                        const T v2 = v2s[r][v];
                        T* q = orow + r * sx + 32 * v;
                        const int ox = oxv[v], oy = oyr[r];
                        *q = v2;
                        if (ox) q[ox] = v2;
                        if (oy) {
                            q[oy] = v2;
                            if (ox) q[oy + ox] = v2;
                        }
                        if (ez) {
                            T* qz = q + ozv;
                            *qz = v2;
                            if (ox) qz[ox] = v2;
                            if (oy) {
                                qz[oy] = v2;
                                if (ox) qz[oy + ox] = v2;
                            }
                        }
                    }
                }
                orow += Sz;
                }
            }
#pragma unroll
            for (int r = 0; r < RG; r++)
#pragma unroll
                for (int v = 0; v < PV; v++) {
                    ro2[r][v] = rn[r][v];
                    if constexpr (HELM) ao2[r][v] = an[r][v];
                }
            sc = sn;
            if (++sn == nst) {
                sn = 0;
                pn ^= 1;
            }
            return true;
        };
        const int nsteps = nzl + 2;
        if (consumers_any(!ok, SH::NC)) return;
        for (int t = 0; t < nsteps; t += 3) {
            if (!step(std::integral_constant<int, 0>{}, t)) break;
            if (t + 1 >= nsteps || !step(std::integral_constant<int, 1>{}, t + 1)) break;
            if (t + 2 >= nsteps || !step(std::integral_constant<int, 2>{}, t + 2)) break;
        }
        if constexpr (NORM) warp_max_atomic(m, a.result);
    };
    if (g == 0) run(std::integral_constant<int, 0>{});
    else run(std::integral_constant<int, 1>{});
}

// Smallest x segment width (elements) of a row copy: a multiple of 128 bytes (every shared-memory
// destination stays 128-byte aligned) with nb segments covering the grown pitch sx, each <= 256.
inline void relax2_segments(int sx, int esize, int* nb, int* bw)
{
    const int q = 128 / esize;
    int b = (sx + 255) / 256;
    int w = ((sx + b - 1) / b + q - 1) / q * q;
    while (w > 256) {
        b++;
        w = ((sx + b - 1) / b + q - 1) / q * q;
    }
    *nb = b;
    *bw = w;
}

} // namespace pb
