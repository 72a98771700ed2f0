// Star-shaped stencil kernels (terms only on the axes, |offset| <= R) for sm_100a.
//
// Two kernels share the same epilogue interface:
//   k_star_tma    : TMA-staged z-streaming. A CTA owns a 64 x TY column of output points and a
//                   chunk of z; planes of the source tile (with an R-wide halo in x and y) arrive
//                   in shared memory through cp.async.bulk.tensor into an NST-deep ring guarded by
//                   mbarriers, z-neighbours live in a (2R+1)-register window per thread, x/y
//                   neighbours are read from the centre plane in shared memory.
//   k_star_simple : one thread per point, read-only cached global loads (small boxes, and any
//                   box the TMA alignment rules exclude).
//
// Terms are evaluated in the stencil's insertion order with one rounding per multiply and per add
// (no FMA), so the result is bitwise the reference's Stencil::hostApply
// (include/base/implem/Proto_StencilImplem.H:725-828 in the reference project).
#pragma once
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

// Geometry of one star application. Index-box point (x,y,z), 0 <= x < nx ..., maps to source-local
// coordinates (x+ox, y+oy, z+oz) in a field of extents (Sx, Sy, Sz).
struct StarGeom {
    int nx, ny, nz;
    int ox, oy, oz;
    int Sx, Sy, Sz;
    int zc;     // z chunk per CTA (TMA kernel)
    int pad;    // TMA kernel: smem x offset of the halo start
};

constexpr int kStarTX = 64;

template <class S, typename T, int TY>
struct StarSmem {
    static constexpr int EV = 16 / (int)sizeof(T);                  // elements per 16 bytes
    static constexpr int BX = ((kStarTX + 2 * S::R + (EV - 1)) + EV - 1) / EV * EV;
    static constexpr int BY = TY + 2 * S::R;
    static constexpr int PLANE_TX = BX * BY * (int)sizeof(T);       // bytes one TMA box delivers
    static constexpr int PLANE = (PLANE_TX + 127) / 128 * 128;
};

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

template <class S, typename T, int TY, int NST, class Epi>
__global__ void __launch_bounds__(kStarTX * TY)
    k_star_tma(const __grid_constant__ CUtensorMap tmap, const StarGeom g, const Coefs<T> cf, const Epi epi_in)
{
    using SM = StarSmem<S, T, TY>;
    constexpr int R = S::R;
    static_assert(NST >= 2 * R + 1, "ring must hold the whole z window");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + NST * SM::PLANE);
    __shared__ int s_abort;
    __shared__ int s_issued;     // planes whose TMA copy has been issued (written by thread 0)

    Epi epi = epi_in;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kStarTX + tx;
    const int x0 = blockIdx.x * kStarTX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * g.zc;
    const int nzl = min(g.zc, g.nz - zb);
    if (nzl <= 0) return;
    const int nplanes = nzl + 2 * R;
    const int xs = g.ox + x0 - R - g.pad;            // 16-byte aligned element coordinate
    const int ys = g.oy + y0 - R;
    const int zs0 = g.oz + zb - R;
    const int x = x0 + tx, y = y0 + ty;
    const bool active = (x < g.nx) && (y < g.ny);
    const int sc = (ty + R) * SM::BX + (tx + R + g.pad);   // centre element inside a plane

    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < NST; s++) mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        int np = nplanes < NST ? nplanes : NST;
        for (int q = 0; q < np; q++) {
            mbar_arrive_expect_tx(&bars[q], SM::PLANE_TX);
            tma_load_3d(smem_raw + q * SM::PLANE, &tmap, &bars[q], xs, ys, zs0 + q);
        }
        s_issued = np;
    }
    int qpending = 0;   // first plane not yet consumed
    auto plane = [&](int q) -> const T* { return reinterpret_cast<const T*>(smem_raw + (q % NST) * SM::PLANE); };

    T win[2 * R + 1];
    bool ok = true;
#pragma unroll
    for (int q = 0; q < 2 * R; q++) {
        ok &= mbar_wait(&bars[q % NST], (q / NST) & 1);
        win[q] = plane(q)[sc];
    }
    if (!ok) s_abort = 1;
    __syncthreads();
    if (s_abort) goto drain;
    qpending = 2 * R;
    // planes 0..R-1 only fed the window: recycle their slots
    if (tid == 0) {
        for (int q = 0; q < R; q++) {
            int nq = q + NST;
            if (nq < nplanes) {
                mbar_arrive_expect_tx(&bars[nq % NST], SM::PLANE_TX);
                tma_load_3d(smem_raw + (nq % NST) * SM::PLANE, &tmap, &bars[nq % NST], xs, ys, zs0 + nq);
                s_issued = nq + 1;
            }
        }
    }

    for (int zo = 0; zo < nzl; zo++) {
        const int qn = zo + 2 * R, qc = zo + R;
        qpending = qn;
        if (!mbar_wait(&bars[qn % NST], (qn / NST) & 1)) s_abort = 1;
        win[2 * R] = plane(qn)[sc];
        const T* pc = plane(qc);
        const int z = zb + zo;
        T acc = epi.init(x, y, z, active);
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const int ox = S::off(j, 0), oy = S::off(j, 1), oz = S::off(j, 2);
            T v;
            if (oz != 0) v = win[R + oz];
            else if (ox == 0 && oy == 0) v = win[R];
            else v = pc[sc + oy * SM::BX + ox];
            acc = dadd(acc, dmul(cf.c[j], v));
        }
        if (active) epi.finish(x, y, z, acc, win[R]);
#pragma unroll
        for (int k = 0; k < 2 * R; k++) win[k] = win[k + 1];
        __syncthreads();
        if (s_abort) goto drain;
        if (tid == 0) {
            int nq = qc + NST;
            if (nq < nplanes) {
                mbar_arrive_expect_tx(&bars[nq % NST], SM::PLANE_TX);
                tma_load_3d(smem_raw + (nq % NST) * SM::PLANE, &tmap, &bars[nq % NST], xs, ys, zs0 + nq);
                s_issued = nq + 1;
            }
        }
    }
    epi.end();
    return;

drain:
    // a wait expired: give the copies still in flight a bounded chance to land, then leave
    if (tid == 0) {
        for (int q = qpending; q < s_issued; q++) {
            for (uint32_t i = 0; i < kMaxWaitTries; i++)
                if (mbar_try_wait(&bars[q % NST], (q / NST) & 1)) break;
        }
    }
    __syncthreads();
}

template <class S, typename T, class Epi>
__global__ void __launch_bounds__(256) k_star_simple(const T* __restrict__ src, const StarGeom g, const Coefs<T> cf,
                                                     const Epi epi_in)
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
        T acc = epi.init(x, y, z, true);
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const long long o = S::off(j, 0) + Sx * S::off(j, 1) + Sxy * S::off(j, 2);
            acc = dadd(acc, dmul(cf.c[j], __ldg(src + base + o)));
        }
        epi.finish(x, y, z, acc, __ldg(src + base));
    }
    epi.end();
}

// ---- basic epilogues ---------------------------------------------------------------------------
// Output addressing for a field on a box: index-box point (x,y,z) -> (x+dx) + Dx*(y+dy) + Dxy*(z+dz)
struct OutMap {
    long long dx, dy, dz, Dx, Dxy;
    __device__ __forceinline__ long long at(int x, int y, int z) const { return (x + dx) + Dx * (y + dy) + Dxy * (z + dz); }
};

// "dst |= S(src)" (init 0) and "dst += S(src)" (init = old dst value, then the terms)
template <typename T>
struct EpiStore {
    T* dst;
    OutMap m;
    int accumulate;
    __device__ __forceinline__ T init(int x, int y, int z, bool active) const
    {
        return (accumulate && active) ? dst[m.at(x, y, z)] : T(0);
    }
    __device__ __forceinline__ void finish(int x, int y, int z, T acc, T) const { dst[m.at(x, y, z)] = acc; }
    __device__ __forceinline__ void end() const {}
};

// out = a*Lu + b*u  /  out = u + a*Lu
template <typename T>
struct EpiAxpby {
    T* dst;
    OutMap m;
    T a, b;
    int euler;
    __device__ __forceinline__ T init(int, int, int, bool) const { return T(0); }
    __device__ __forceinline__ void finish(int x, int y, int z, T acc, T u) const
    {
        dst[m.at(x, y, z)] = euler ? dadd(u, dmul(a, acc)) : dadd(dmul(a, acc), dmul(b, u));
    }
    __device__ __forceinline__ void end() const {}
};

} // namespace pb
