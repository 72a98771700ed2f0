// Device side of the periodic multigrid: grown-level layout, periodic image stores, the smoother,
// residual/restriction/prolongation kernels, the star-kernel epilogues of the fused passes and the
// single-CTA coarse cycle. Shared by the single-solve solver (pb_mg.cu) and the serving engine
// (pb_serve.cu), so both run the same per-cell arithmetic.
#pragma once
#include <cstring>
#include <type_traits>

#include "pb_internal.cuh"
#include "pb_star.cuh"

namespace pb {

// A level is one periodic n^3 box held with a one-cell ghost layer: cell (x, y, z), -1 <= x,y,z <= n,
// sits at (x+1) + sx*((y+1) + (n+2)*(z+1)). The x pitch sx >= n+2 is n+2 rounded up to 16 bytes,
// so every row starts on a 16-byte boundary (a TMA requirement); columns past n+1 are padding.
template <typename T>
constexpr int grown_pitch(int n)
{
    return (n + 2 + (16 / (int)sizeof(T)) - 1) / (16 / (int)sizeof(T)) * (16 / (int)sizeof(T));
}

// Writes v to the valid cell (x,y,z) and to every ghost cell that is a periodic image of it.
// Out of line: only cells on the box boundary call it, and keeping its index arrays out of the
// fused stencil kernels keeps their register count low.
template <typename T>
__device__ __noinline__ void store_periodic_images(T* out, int n, int sx, int x, int y, int z, T v)
{
    const long long Sy = sx, Sz = (long long)sx * (n + 2);
    int xs[3], ys[3], zs[3];
    int nx = 1, ny = 1, nz = 1;
    xs[0] = x + 1;
    ys[0] = y + 1;
    zs[0] = z + 1;
    if (x == 0) xs[nx++] = n + 1;
    if (x == n - 1) xs[nx++] = 0;
    if (y == 0) ys[ny++] = n + 1;
    if (y == n - 1) ys[ny++] = 0;
    if (z == 0) zs[nz++] = n + 1;
    if (z == n - 1) zs[nz++] = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) out[xs[i] + Sy * ys[j] + Sz * zs[k]] = v;
}

template <typename T>
__device__ __forceinline__ long long grown_index(int n, int sx, int x, int y, int z)
{
    return (x + 1) + (long long)sx * ((y + 1) + (long long)(n + 2) * (z + 1));
}

// Which periodic image of a coordinate exists: 0 none, 1 at +n (c == 0), 2 at -n (c == n-1).
__device__ __forceinline__ int edge_code(int c, int n) { return c == 0 ? 1 : (c == n - 1 ? 2 : 0); }

// Writes v at q (the valid cell) and at its periodic images, given the edge codes of x, y, z. The
// images sit at constant offsets +-n, +-n*sx, +-n*sx*(n+2) from q, so this is a few predicated
// stores. n == 1 (a cell that is both first and last) takes the general path.
template <typename T>
__device__ __forceinline__ void store_with_images(T* out, int n, int sx, T* q, int ex, int ey, int ez, T v)
{
    *q = v;
    if ((ex | ey | ez) == 0) return;
    if (n == 1) {
        store_periodic_images(out, n, sx, 0, 0, 0, v);
        return;
    }
    const long long ox = ex == 0 ? 0 : (ex == 1 ? n : -n);
    const long long oy = ey == 0 ? 0 : (ey == 1 ? (long long)n * sx : -(long long)n * sx);
    const long long sz = (long long)n * sx * (n + 2);
    const long long oz = ez == 0 ? 0 : (ez == 1 ? sz : -sz);
    if (ox) q[ox] = v;
    if (oy) q[oy] = v;
    if (ox && oy) q[ox + oy] = v;
    if (oz) {
        q[oz] = v;
        if (ox) q[oz + ox] = v;
        if (oy) q[oz + oy] = v;
        if (ox && oy) q[oz + ox + oy] = v;
    }
}

template <typename T>
__device__ __forceinline__ void store_periodic(T* out, int n, int sx, int x, int y, int z, T v)
{
    store_with_images(out, n, sx, out + grown_index<T>(n, sx, x, y, z), edge_code(x, n), edge_code(y, n),
                      edge_code(z, n), v);
}

// Row cursor of a periodic output for a thread's points x, x+1 (kPV of them) in one row: the
// address of the first point's valid cell at the row's first plane z0, and the constant offsets of
// the periodic images (0 when there is none): per point in x, and for the row in y.
constexpr int kPV = 2;
template <typename T>
struct PeriodicRow {
    T* p;
    int z0;
    int yo;
    int xo[kPV];
    bool act;
    __device__ __forceinline__ bool active() const { return act; }
};
__device__ __forceinline__ int image_offset(int c, int n, int stride)
{
    return c == 0 ? n * stride : (c == n - 1 ? -n * stride : 0);
}
template <typename T>
__device__ __forceinline__ PeriodicRow<T> periodic_row(T* out, int n, int sx, int x, int y, int z0, bool active)
{
    PeriodicRow<T> r;
    r.p = active ? out + grown_index<T>(n, sx, x, y, z0) : out;
    r.z0 = z0;
    r.act = active;
    r.yo = image_offset(y, n, sx);
#pragma unroll
    for (int v = 0; v < kPV; v++) r.xo[v] = image_offset(x + v, n, 1);
    return r;
}
// Stores v at point (row, plane z0+zo, x+pv) and at its periodic images. ZE: the plane is the
// first or last of the domain. A 1-cell box (every coordinate both first and last) takes the
// general path.
template <bool ZE, typename T>
__device__ __forceinline__ void store_row(T* out, int n, int sx, const PeriodicRow<T>& r, int zo, int pv, T val)
{
    T* q = r.p + (long long)zo * sx * (n + 2) + pv;
    if (n == 1) {
        store_periodic_images(out, n, sx, 0, 0, 0, val);
        return;
    }
    const int xo = r.xo[pv], yo = r.yo;
    *q = val;
    if (xo) q[xo] = val;
    if (yo) {
        q[yo] = val;
        if (xo) q[yo + xo] = val;
    }
    if constexpr (ZE) {
        const long long zs = (long long)n * sx * (n + 2);
        T* qz = q + (r.z0 + zo == 0 ? zs : -zs);
        *qz = val;
        if (xo) qz[xo] = val;
        if (yo) {
            qz[yo] = val;
            if (xo) qz[yo + xo] = val;
        }
    }
}
template <typename T>
__device__ __forceinline__ T load_row(const PeriodicRow<T>& r, int n, int sx, int zo, int pv)
{
    return r.p[(long long)zo * sx * (n + 2) + pv];
}

// Scalars of one level's smoother.
template <typename T>
struct RelaxCoef {
    int n, sx;           // edge and x pitch of the level
    int helm;
    T neg_lambda;        // Poisson form: -omega*h*h/6
    T beta, omega, diagB;
};

// One Jacobi sweep value from the stencil sum acc (L(phi, omega/6) for the Poisson form,
// L(phi, 1/h^2) for the Helmholtz form), the centre value c, rho and alpha.
template <typename T>
__device__ __forceinline__ T relax_value(const RelaxCoef<T>& k, T acc, T c, T rho, T al)
{
    if (!k.helm) return dadd(c, dmadd(acc, k.neg_lambda, rho));
    const T r = dsub(rho, dsub(dmul(al, c), dmul(k.beta, acc)));
    return dadd(c, squot(dmul(k.omega, r), dadd(al, k.diagB)));
}

// relax epilogue: auxiliary field 0 = rho, 1 = alpha (Helmholtz)
template <typename T>
struct EpiRelax {
    T* out;
    RelaxCoef<T> k;
    using Row = PeriodicRow<T>;
    static constexpr bool kZEdge = true;
    static constexpr int kAux = 2;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const { return periodic_row(out, k.n, k.sx, x, y, z0, active); }
    __device__ __forceinline__ bool z_edge(int z) const { return z == 0 || z == k.n - 1; }
    __device__ __forceinline__ T init(const Row&, int, int, const AuxCtx&) const { return T(0); }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int pv, T acc, T c, const AuxCtx& ax) const
    {
        if (!r.active()) return;
        const T al = k.helm ? ax.get<T>(1) : T(0);
        store_row<ZE>(out, k.n, k.sx, r, zo, pv, relax_value(k, acc, c, ax.get<T>(0), al));
    }
    __device__ __forceinline__ void end_warp() const {}
    __device__ __forceinline__ void end_block() const {}
};

// Last FP32 post-smoothing sweep of a mixed-precision cycle, fused with the FP64 correction:
// u64 += (double) e_new, periodic images included. Auxiliary fields 0 = u64 itself (its old value
// arrives through the pipeline instead of a dependent load), 1 = rho, 2 = alpha (Helmholtz).
struct EpiRelaxUpdate {
    double* u;
    int usx;             // x pitch of u
    RelaxCoef<float> k;
    using Row = PeriodicRow<double>;
    static constexpr bool kZEdge = true;
    static constexpr int kAux = 3;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const { return periodic_row(u, k.n, usx, x, y, z0, active); }
    __device__ __forceinline__ bool z_edge(int z) const { return z == 0 || z == k.n - 1; }
    __device__ __forceinline__ float init(const Row&, int, int, const AuxCtx&) const { return 0.f; }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int pv, float acc, float c, const AuxCtx& ax) const
    {
        if (!r.active()) return;
        const float al = k.helm ? ax.get<float>(2) : 0.f;
        const float e = relax_value(k, acc, c, ax.get<float>(1), al);
        store_row<ZE>(u, k.n, usx, r, zo, pv, dadd(ax.get<double>(0), (double)e));
    }
    __device__ __forceinline__ void end_warp() const {}
    __device__ __forceinline__ void end_block() const {}
};

// residual max-norm epilogue: Poisson acc starts at (0 - rho) with L(phi, 1/h^2); Helmholtz
// r = rho - (alpha*phi - beta*L(phi, 1/h^2)). Auxiliary fields as in EpiRelax.
template <typename T>
struct EpiResnorm {
    int helm;
    T beta;
    double* result;
    double m;
    using Row = OutRow<T>;
    static constexpr bool kZEdge = false;
    static constexpr int kAux = 2;
    __device__ __forceinline__ Row row(int, int, int, bool active) const { return Row{nullptr, active}; }
    __device__ __forceinline__ bool z_edge(int) const { return false; }
    __device__ __forceinline__ T init(const Row& r, int, int, const AuxCtx& ax) const
    {
        if (helm || !r.active) return T(0);
        return dsub(T(0), ax.get<T>(0));
    }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int, int, T acc, T c, const AuxCtx& ax)
    {
        if (!r.active) return;
        if (!helm) {
            m = upd_abs(m, (double)acc);
        } else {
            const T res = dsub(ax.get<T>(0), dsub(dmul(ax.get<T>(1), c), dmul(beta, acc)));
            m = upd_abs(m, (double)res);
        }
    }
    __device__ __forceinline__ void end_warp() const { warp_max_atomic(m, result); }
    __device__ __forceinline__ void end_block() const { block_max_atomic(m, result); }
};

// A Jacobi sweep fused with the max-norm residual of the state it reads: the norm the solver tests
// after a cycle is taken during the next cycle's first sweep (the sweep writes the other buffer,
// so the state measured stays intact for the caller if it has converged). acc is the smoother's
// sum (relax_value, as EpiRelax), acc2 the operator's: (0 - f) + L(u, 1/h^2) for the Poisson form,
// L(u, 1/h^2) for the Helmholtz form, both in the Laplacian's term order, so the norm is bitwise
// EpiResnorm's. Auxiliary fields: 0 = rho (= f), 1 = alpha (Helmholtz).
template <typename T>
struct EpiRelaxNorm {
    T* out;
    RelaxCoef<T> k;
    Coefs<T> c2;         // L(., 1/h^2)
    T beta;
    double* result;
    double m;
    using Row = PeriodicRow<T>;
    static constexpr bool kZEdge = true;
    static constexpr bool kTwoSums = true;
    static constexpr int kAux = 2;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const { return periodic_row(out, k.n, k.sx, x, y, z0, active); }
    __device__ __forceinline__ bool z_edge(int z) const { return z == 0 || z == k.n - 1; }
    __device__ __forceinline__ T init(const Row&, int, int, const AuxCtx&) const { return T(0); }
    __device__ __forceinline__ T init2(const Row& r, int, int, const AuxCtx& ax) const
    {
        if (k.helm || !r.active()) return T(0);
        return dsub(T(0), ax.get<T>(0));
    }
    template <bool ZE>
    __device__ __forceinline__ void finish2(const Row& r, int zo, int pv, T acc, T acc2, T c, const AuxCtx& ax)
    {
        if (!r.active()) return;
        const T rho = ax.get<T>(0);
        const T al = k.helm ? ax.get<T>(1) : T(0);
        store_row<ZE>(out, k.n, k.sx, r, zo, pv, relax_value(k, acc, c, rho, al));
        if (!k.helm) m = upd_abs(m, (double)acc2);
        else m = upd_abs(m, (double)dsub(rho, dsub(dmul(al, c), dmul(beta, acc2))));
    }
    __device__ __forceinline__ void end_warp() const { warp_max_atomic(m, result); }
    __device__ __forceinline__ void end_block() const { block_max_atomic(m, result); }
};

// Mixed precision, one pass over the FP64 state u (auxiliary fields: 0 = f, 1 = alpha):
//   r = (0 + f) + L(u, -1/h^2)  |  r = f - (alpha*u - beta*L(u, 1/h^2))   (FP64)
//   norm = max |r|; rhs32 = float(r); first FP32 sweep of the next cycle from e = 0 into e32.
struct Res64Row {
    PeriodicRow<float> e;
    float* r;
};
struct EpiRes64 {
    float* e32;          // grown FP32 level (pitch k.sx); null: no first sweep (the cycle starts
                         // with a two-sweep pass from zero)
    float* rhs32;        // n^3
    int helm;
    double beta;
    RelaxCoef<float> k;
    double* result;
    double m;
    using Row = Res64Row;
    static constexpr bool kZEdge = true;
    static constexpr int kAux = 2;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const
    {
        Row r;
        r.e = periodic_row(e32 ? e32 : rhs32, k.n, k.sx, x, y, z0, active);   // rhs32: a valid base, never stored through
        r.r = active ? rhs32 + x + (long long)k.n * (y + (long long)k.n * z0) : rhs32;
        return r;
    }
    __device__ __forceinline__ bool z_edge(int z) const { return z == 0 || z == k.n - 1; }
    __device__ __forceinline__ double init(const Row& r, int, int, const AuxCtx& ax) const
    {
        if (helm || !r.e.active()) return 0.0;
        return dadd(0.0, ax.get<double>(0));
    }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int pv, double acc, double c, const AuxCtx& ax)
    {
        if (!r.e.active()) return;
        double res = acc;
        float al = 0.f;
        if (helm) {
            const double a64 = ax.get<double>(1);
            res = dsub(ax.get<double>(0), dsub(dmul(a64, c), dmul(beta, acc)));
            al = __double2float_rn(a64);
        }
        m = upd_abs(m, res);
        const float r32 = __double2float_rn(res);
        r.r[(long long)zo * k.n * k.n + pv] = r32;
        if (e32) store_row<ZE>(e32, k.n, k.sx, r.e, zo, pv, relax_value(k, 0.f, 0.f, r32, al));
    }
    __device__ __forceinline__ void end_warp() const { warp_max_atomic(m, result); }
    __device__ __forceinline__ void end_block() const { block_max_atomic(m, result); }
};

// first sweep from phi == 0 (every read of phi would return +0.0)
template <typename T>
__global__ void __launch_bounds__(256) k_relax_first(const T* __restrict__ rhs, const T* __restrict__ alpha, T* out,
                                                     RelaxCoef<T> k)
{
    const int n = k.n;
    const long long total = (long long)n * n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % n);
        long long q = i / n;
        int y = (int)(q % n), z = (int)(q / n);
        const T al = k.helm ? alpha[i] : T(0);
        store_periodic(out, n, k.sx, x, y, z, relax_value(k, T(0), T(0), rhs[i], al));
    }
}

// exact coarsest-level solve: out = Ainv * rhs (one thread per cell, products summed in column order)
template <typename T>
__global__ void __launch_bounds__(256) k_bottom_direct(const T* __restrict__ ainv, const T* __restrict__ rhs, T* out,
                                                       int n, int sx)
{
    const int N = n * n * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        T acc = T(0);
        for (int j = 0; j < N; j++) acc = dmadd(acc, ainv[(long long)i * N + j], rhs[j]);
        store_periodic(out, n, sx, i % n, (i / n) % n, i / (n * n), acc);
    }
}

static __global__ void __launch_bounds__(256) k_to_float(const double* __restrict__ a, float* b, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = __double2float_rn(a[i]);
}

// One fine cell's residual for the restriction: rho + L(phi, -1/h^2) (Poisson form, cf scaled by
// -1/h^2) or rho - (alpha*phi - beta*L(phi, 1/h^2)) (Helmholtz form, cf scaled by 1/h^2).
template <typename T>
__device__ __forceinline__ T fine_residual(const T* phi, long long gi, long long Sy, long long Sz, T rho, T al,
                                           int helm, const Coefs<T>& cf, T beta)
{
    if (!helm) {
        T r = dadd(T(0), rho);
#pragma unroll
        for (int j = 0; j < ShapeLap7::NT; j++) {
            const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
            r = dmadd(r, cf.c[j], phi[gi + o]);
        }
        return r;
    }
    T lp = T(0);
#pragma unroll
    for (int j = 0; j < ShapeLap7::NT; j++) {
        const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
        lp = dmadd(lp, cf.c[j], phi[gi + o]);
    }
    return dsub(rho, dsub(dmul(al, phi[gi]), dmul(beta, lp)));
}

// coarse right-hand side: AvgDown(2) of the fine residual, children in Box([0,1]^3) order.
// Block (32, 8): one thread per coarse cell of a (cx, cy) tile; blockIdx.z = cz.
template <typename T>
__global__ void __launch_bounds__(256) k_resid_restrict(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                        const T* __restrict__ alpha, T* rhs_c, int nf, int sx, int helm,
                                                        Coefs<T> cf, T beta)
{
    const int nc = nf / 2;
    const int cx = blockIdx.x * 32 + threadIdx.x, cy = blockIdx.y * 8 + threadIdx.y, cz = blockIdx.z;
    if (cx >= nc || cy >= nc) return;
    const long long Sy = sx, Sz = (long long)sx * (nf + 2);
    const T eighth = T(1.0 / 8);
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int fx = 2 * cx + (k & 1), fy = 2 * cy + ((k >> 1) & 1), fz = 2 * cz + (k >> 2);
        const long long fi = fx + (long long)nf * (fy + (long long)nf * fz);
        const T al = helm ? __ldg(alpha + fi) : T(0);
        const T r = fine_residual(phi, grown_index<T>(nf, sx, fx, fy, fz), Sy, Sz, __ldg(rhs + fi), al, helm, cf, beta);
        acc = dmadd(acc, eighth, r);
    }
    rhs_c[cx + (long long)nc * (cy + (long long)nc * cz)] = acc;
}
static inline dim3 restrict_grid(int nf) { return dim3((nf / 2 + 31) / 32, (nf / 2 + 7) / 8, nf / 2); }

// The same coarse right-hand side through the TMA-staged star kernel (k_star_tma with two x points
// in each of two rows per thread, chunks of an even number of planes starting on an even plane):
// a thread's four points of a plane are the children (dx, dy) of one coarse cell and two
// consecutive planes its dz = 0, 1, so the kernel hands the eight fine residuals of a coarse cell to
// the same thread in Box([0,1]^3) order (x fastest). Each residual is fine_residual's arithmetic
// (the star kernel sums the taps in the Laplacian's order from init's start value) and the eight
// are summed as 1/8 each in that order, as k_resid_restrict does.
template <typename T>
struct EpiRestrict {
    T* rhs_c;            // coarse right-hand side (nc^3)
    int nc;
    int helm;
    T beta;
    T sum;               // running sum of the thread's current coarse cell
    struct Row {
        T* out;          // the coarse cell under this point at the chunk's first coarse plane
        int dy;          // child row (y & 1)
        bool act;
        __device__ __forceinline__ bool active() const { return act; }
    };
    static constexpr bool kZEdge = false;
    static constexpr int kAux = 2;
    __device__ __forceinline__ Row row(int x, int y, int z0, bool active) const
    {
        Row w;
        w.dy = y & 1;
        w.act = active;
        w.out = active ? rhs_c + (x >> 1) + (long long)nc * ((y >> 1) + (long long)nc * (z0 >> 1)) : rhs_c;
        return w;
    }
    __device__ __forceinline__ bool z_edge(int) const { return false; }
    __device__ __forceinline__ T init(const Row& r, int, int, const AuxCtx& ax) const
    {
        if (helm || !r.act) return T(0);
        return dadd(T(0), ax.get<T>(0));
    }
    template <bool ZE>
    __device__ __forceinline__ void finish(const Row& r, int zo, int v, T acc, T c, const AuxCtx& ax)
    {
        const int child = v + 2 * r.dy + 4 * (zo & 1);
        if (child == 0) sum = T(0);
        if (!r.act) return;
        T res = acc;
        if (helm) res = dsub(ax.get<T>(0), dsub(dmul(ax.get<T>(1), c), dmul(beta, acc)));
        sum = dmadd(sum, T(1.0 / 8), res);
        if (child == 7) r.out[(long long)(zo >> 1) * nc * nc] = sum;
    }
    __device__ __forceinline__ void end_warp() const {}
    __device__ __forceinline__ void end_block() const {}
};

// The same coarse right-hand side, marching in z. Block (32, 8): lane = fine x (32 consecutive
// fine cells, coalesced), threadIdx.y = coarse row cy (fine rows 2cy, 2cy+1); the block walks
// coarse planes [cz0, cz0 + czc). Each fine row keeps phi at the fine planes 2cz-1 .. 2cz+2 in a
// register window (two new planes per coarse plane), and the y taps between the thread's two rows
// come from registers, so a fine cell costs about five loads instead of eight. Each fine residual
// is fine_residual's arithmetic (taps in the Laplacian's order); the even lane of a pair gathers
// its neighbour's four residuals by shuffle and sums the eight children in Box([0,1]^3) order.
template <typename T>
__global__ void __launch_bounds__(256) k_resid_restrict_z(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                          const T* __restrict__ alpha, T* rhs_c, int nf, int sx,
                                                          int helm, Coefs<T> cf, T beta, int czc)
{
    const int nc = nf / 2;
    const int fx = blockIdx.x * 32 + threadIdx.x, cy = blockIdx.y * 8 + threadIdx.y;
    const int cz0 = blockIdx.z * czc, cz1 = min(cz0 + czc, nc);
    const bool act = fx < nf && cy < nc;          // warp-uniform in y; x lanes beyond nf idle
    const long long Sy = sx, Sz = (long long)sx * (nf + 2);
    const T eighth = T(1.0 / 8);
    const int fy0 = 2 * cy;
    // grown address of (fx, fy0, fz) = base + fz * Sz; rows fy0 and fy0 + 1
    const T* base = phi + (act ? grown_index<T>(nf, sx, fx, fy0, 0) : 0);
    T w[2][4];                                    // [row][fine plane 2cz-1 .. 2cz+2]
    if (act) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            w[r][2] = base[r * Sy + (long long)(2 * cz0 - 1) * Sz];
            w[r][3] = base[r * Sy + (long long)(2 * cz0) * Sz];
        }
    }
    for (int cz = cz0; cz < cz1; cz++) {
        T res[2][2];                              // [row][fine plane 2cz, 2cz+1]
        if (act) {
#pragma unroll
            for (int r = 0; r < 2; r++) {
                w[r][0] = w[r][2];
                w[r][1] = w[r][3];
                w[r][2] = base[r * Sy + (long long)(2 * cz + 1) * Sz];
                w[r][3] = base[r * Sy + (long long)(2 * cz + 2) * Sz];
            }
#pragma unroll
            for (int pz = 0; pz < 2; pz++) {
                const int fz = 2 * cz + pz;
#pragma unroll
                for (int r = 0; r < 2; r++) {
                    const T* q = base + r * Sy + (long long)fz * Sz;
                    const long long fi = fx + (long long)nf * ((fy0 + r) + (long long)nf * fz);
                    const T c = w[r][pz + 1];
                    // taps in the Laplacian's order: 0, +x, -x, +y, -y, +z, -z
                    const T t[7] = {c, q[1], q[-1], r == 0 ? w[1][pz + 1] : q[Sy], r == 1 ? w[0][pz + 1] : q[-Sy],
                                    w[r][pz + 2], w[r][pz]};
                    const T rho = __ldg(rhs + fi);
                    if (!helm) {
                        T v = dadd(T(0), rho);
#pragma unroll
                        for (int j = 0; j < 7; j++) v = dmadd(v, cf.c[j], t[j]);
                        res[r][pz] = v;
                    } else {
                        T lp = T(0);
#pragma unroll
                        for (int j = 0; j < 7; j++) lp = dmadd(lp, cf.c[j], t[j]);
                        res[r][pz] = dsub(rho, dsub(dmul(__ldg(alpha + fi), c), dmul(beta, lp)));
                    }
                }
            }
        } else {
            res[0][0] = res[0][1] = res[1][0] = res[1][1] = T(0);
        }
        // children k = dx + 2 dy + 4 dz; dx = 1 lives in the odd lane
        T odd[2][2];
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int pz = 0; pz < 2; pz++) odd[r][pz] = __shfl_down_sync(0xffffffffu, res[r][pz], 1);
        if (act && (fx & 1) == 0) {
            T acc = T(0);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
                acc = dmadd(acc, eighth, dx ? odd[dy][dz] : res[dy][dz]);
            }
            rhs_c[fx / 2 + (long long)nc * (cy + (long long)nc * cz)] = acc;
        }
    }
}
// The same restriction with x pairs: lane = coarse x, so a thread's fine columns 2cx and 2cx+1 (a
// coarse cell's x children) and their x neighbours 2cx-1 and 2cx+2 come from two aligned 2-wide
// loads per row and plane (grown x index 2cx is even and rows start 16-byte aligned), a warp covers
// 64 consecutive fine cells, and no shuffle is needed. Block (32, 8) = 32 coarse x by 8 coarse rows;
// the block walks coarse planes [cz0, cz0 + czc) with the register window of k_resid_restrict_z.
// Same taps, same order, same child sum: bitwise that kernel's results. Needs nf even, nf >= 64.
template <typename T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };
template <typename T>
__global__ void __launch_bounds__(256) k_resid_restrict_x2(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                           const T* __restrict__ alpha, T* rhs_c, int nf, int sx,
                                                           int helm, Coefs<T> cf, T beta, int czc)
{
    using P2 = typename Pair<T>::type;
    const int nc = nf / 2;
    const int cx = blockIdx.x * 32 + threadIdx.x, cy = blockIdx.y * 8 + threadIdx.y;
    const int cz0 = blockIdx.z * czc, cz1 = min(cz0 + czc, nc);
    const bool act = cx < nc && cy < nc;
    const long long Sy = sx, Sz = (long long)sx * (nf + 2);
    const T eighth = T(1.0 / 8);
    const int fx = 2 * cx, fy0 = 2 * cy;
    // fine (fx - 1, fy0, 0): the first element of an aligned pair
    const T* base = phi + (act ? grown_index<T>(nf, sx, fx - 1, fy0, 0) : 0);
    T w[2][4][4];                                 // [row][fine plane 2cz-1 .. 2cz+2][fine x fx-1 .. fx+2]
    auto load4 = [&](T* d, const T* q) {
        const P2 a = *reinterpret_cast<const P2*>(q), b = *reinterpret_cast<const P2*>(q + 2);
        d[0] = a.x;
        d[1] = a.y;
        d[2] = b.x;
        d[3] = b.y;
    };
    if (act) {
#pragma unroll
        for (int r = 0; r < 2; r++) {
            load4(w[r][2], base + r * Sy + (long long)(2 * cz0 - 1) * Sz);
            load4(w[r][3], base + r * Sy + (long long)(2 * cz0) * Sz);
        }
    }
    for (int cz = cz0; cz < cz1; cz++) {
        if (!act) continue;
#pragma unroll
        for (int r = 0; r < 2; r++) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                w[r][0][i] = w[r][2][i];
                w[r][1][i] = w[r][3][i];
            }
            load4(w[r][2], base + r * Sy + (long long)(2 * cz + 1) * Sz);
            load4(w[r][3], base + r * Sy + (long long)(2 * cz + 2) * Sz);
        }
        T res[2][2][2];                           // [row][fine plane 2cz, 2cz+1][dx]
#pragma unroll
        for (int pz = 0; pz < 2; pz++) {
            const int fz = 2 * cz + pz;
            // the rows beyond the thread's two: fy0 - 1 and fy0 + 2 at (fx, fx + 1)
            const T* qm = base + 1 - Sy + (long long)fz * Sz;
            const T* qp = base + 1 + 2 * Sy + (long long)fz * Sz;
            const T om[2] = {qm[0], qm[1]}, op[2] = {qp[0], qp[1]};
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const long long fi = fx + (long long)nf * ((fy0 + r) + (long long)nf * fz);
                const P2 rr = *reinterpret_cast<const P2*>(rhs + fi);
                P2 aa;
                if (helm) aa = *reinterpret_cast<const P2*>(alpha + fi);
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const T c = w[r][pz + 1][1 + dx];
                    // taps in the Laplacian's order: 0, +x, -x, +y, -y, +z, -z
                    const T t[7] = {c, w[r][pz + 1][2 + dx], w[r][pz + 1][dx], r == 0 ? w[1][pz + 1][1 + dx] : op[dx],
                                    r == 1 ? w[0][pz + 1][1 + dx] : om[dx], w[r][pz + 2][1 + dx], w[r][pz][1 + dx]};
                    const T rho = dx ? rr.y : rr.x;
                    if (!helm) {
                        T v = dadd(T(0), rho);
#pragma unroll
                        for (int j = 0; j < 7; j++) v = dmadd(v, cf.c[j], t[j]);
                        res[r][pz][dx] = v;
                    } else {
                        T lp = T(0);
#pragma unroll
                        for (int j = 0; j < 7; j++) lp = dmadd(lp, cf.c[j], t[j]);
                        res[r][pz][dx] = dsub(rho, dsub(dmul(dx ? aa.y : aa.x, c), dmul(beta, lp)));
                    }
                }
            }
        }
        // children k = dx + 2 dy + 4 dz
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < 8; k++) acc = dmadd(acc, eighth, res[(k >> 1) & 1][k >> 2][k & 1]);
        rhs_c[cx + (long long)nc * (cy + (long long)nc * cz)] = acc;
    }
}
static inline int restrict_x2_chunk(int nf, int sms)
{
    const int nc = nf / 2;
    const long long bxy = (long long)((nc + 31) / 32) * ((nc + 7) / 8);
    const long long want = (long long)sms * 8;
    int czc = (int)((nc * bxy + want - 1) / want);
    return czc < 1 ? 1 : (czc > nc ? nc : czc);
}
static inline dim3 restrict_x2_grid(int nf, int czc)
{
    return dim3((nf / 2 + 31) / 32, (nf / 2 + 7) / 8, (nf / 2 + czc - 1) / czc);
}

// z chunk: about two waves of 8 blocks per SM
static inline int restrict_z_chunk(int nf, int sms)
{
    const int nc = nf / 2;
    const long long bxy = (long long)((nf + 31) / 32) * ((nc + 7) / 8);
    const long long want = 2LL * sms * 8;
    int czc = (int)((nc * bxy + want - 1) / want);
    return czc < 1 ? 1 : (czc > nc ? nc : czc);
}
static inline dim3 restrict_z_grid(int nf, int czc)
{
    return dim3((nf + 31) / 32, (nf / 2 + 7) / 8, (nf / 2 + czc - 1) / czc);
}

// phi += 1.0 * delta_c(p/2) on the valid box, periodic images included. Block (32, 8): a thread
// takes the eight fine cells x, x + 32 (every warp access 32 consecutive cells) of the two fine rows
// and two fine planes over one coarse row and plane, so two coarse loads serve eight cells and the
// eight fine loads are in flight together before any store.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong(T* phi, const T* __restrict__ delta_c, int nf, int sxf, int sxc)
{
    const int nc = nf / 2;
    const int cy = blockIdx.y * 8 + threadIdx.y, cz = blockIdx.z;
    if (cy >= nc) return;
    const long long Sy = sxf, Sz = (long long)sxf * (nf + 2);
    const T* drow = delta_c + grown_index<T>(nc, sxc, 0, cy, cz);
    T* prow = phi + grown_index<T>(nf, sxf, 0, 2 * cy, 2 * cz);
    T d[2], v[2][2][2];          // [x half][row][plane]
    bool in[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int x = blockIdx.x * 64 + h * 32 + threadIdx.x;
        in[h] = x < nf;
        d[h] = in[h] ? __ldg(drow + x / 2) : T(0);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int pz = 0; pz < 2; pz++) v[h][r][pz] = in[h] ? prow[x + r * Sy + pz * Sz] : T(0);
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (!in[h]) continue;
        const int x = blockIdx.x * 64 + h * 32 + threadIdx.x;
        const int ex = edge_code(x, nf);
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int pz = 0; pz < 2; pz++)
                store_with_images(phi, nf, sxf, prow + x + r * Sy + pz * Sz, ex, edge_code(2 * cy + r, nf),
                                  edge_code(2 * cz + pz, nf), dadd(v[h][r][pz], dmul(T(1), d[h])));
    }
}
static inline dim3 prolong_grid(int nf) { return dim3((nf + 63) / 64, (nf / 2 + 7) / 8, nf / 2); }

// n^3 <-> grown layout with periodic ghost images
template <typename T>
__global__ void __launch_bounds__(256) k_pack_in(const T* __restrict__ src, T* out, int n, int sx)
{
    const long long total = (long long)n * n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % n);
        long long q = i / n;
        store_periodic(out, n, sx, x, (int)(q % n), (int)(q / n), src[i]);
    }
}
template <typename T>
__global__ void __launch_bounds__(256) k_pack_out(const T* __restrict__ g, T* dst, int n, int sx)
{
    const long long total = (long long)n * n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int x = (int)(i % n);
        long long q = i / n;
        dst[i] = g[grown_index<T>(n, sx, x, (int)(q % n), (int)(q / n))];
    }
}

// AvgDown(2) of a plain n^3 field (coarse-level alpha)
template <typename T>
__global__ void __launch_bounds__(256) k_avgdown_plain(const T* __restrict__ f, T* c, int nf)
{
    const int nc = nf / 2;
    const long long total = (long long)nc * nc * nc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int cx = (int)(i % nc);
        long long q = i / nc;
        int cy = (int)(q % nc), cz = (int)(q / nc);
        T acc = T(0);
        for (int k = 0; k < 8; k++) {
            int fx = 2 * cx + (k & 1), fy = 2 * cy + ((k >> 1) & 1), fz = 2 * cz + (k >> 2);
            acc = dadd(acc, dmul(T(1.0 / 8), f[fx + (long long)nf * (fy + (long long)nf * fz)]));
        }
        c[i] = acc;
    }
}


// ---- coarse levels as one kernel ---------------------------------------------------------------
// The levels at and below a small edge run their whole part of the V-cycle inside one CTA: every
// sweep, restriction and prolongation is a block-strided loop followed by __syncthreads, with the
// same per-cell arithmetic (and the same buffer ping-pong) as the one-launch-per-step path, so the
// results are identical; only the launches go away.
constexpr int kMaxCoarse = 8;
constexpr int kCoarseThreads = 1024;
template <typename T>
struct CoarseLevel {
    T* phi[2];
    T* rhs;
    const T* alpha;
    RelaxCoef<T> k;          // n, sx and the smoother's scalars
    Coefs<T> crelax;         // L(., omega/6) (Poisson form) or L(., 1/h^2) (Helmholtz form)
    Coefs<T> cres;           // L(., -1/h^2) (Poisson form) or L(., 1/h^2) (Helmholtz form)
};
template <typename T>
struct CoarseArgs {
    CoarseLevel<T> lv[kMaxCoarse];   // 0 = coarsest
    int top;                         // finest level handled here (entered from zero)
    int nu1, nu2, nu_bottom, direct;
    const T* ainv;
    T beta;
    int in_smem;                     // 1: the levels live in shared memory during the cycle
};

// Shared-memory arena of the coarse cycle: per level two grown buffers, rho and (Helmholtz)
// alpha, each 16-byte aligned. Returns the bytes needed; fills the element offsets when asked.
template <typename T>
static size_t coarse_smem_layout(const CoarseArgs<T>& a, int helm, long long (*off)[4])
{
    size_t total = 0;
    auto take = [&](size_t elems) {
        const size_t o = total;
        total += (elems * sizeof(T) + 15) / 16 * 16;
        return (long long)(o / sizeof(T));
    };
    for (int l = 0; l <= a.top; l++) {
        const CoarseLevel<T>& L = a.lv[l];
        const size_t g = (size_t)L.k.sx * (L.k.n + 2) * (L.k.n + 2), c = (size_t)L.k.n * L.k.n * L.k.n;
        const long long o0 = take(g), o1 = take(g), o2 = take(c), o3 = helm ? take(c) : -1;
        if (off) {
            off[l][0] = o0;
            off[l][1] = o1;
            off[l][2] = o2;
            off[l][3] = o3;
        }
    }
    return total;
}

struct CoarseOffsets {
    long long o[kMaxCoarse][4];      // element offsets of phi0, phi1, rho, alpha per level
};

template <typename T>
__device__ void coarse_relax(const CoarseLevel<T>& L, int cur, bool first)
{
    const int n = L.k.n, sx = L.k.sx;
    const long long Sy = sx, Sz = (long long)sx * (n + 2);
    const T* src = L.phi[cur];
    T* dst = L.phi[1 - cur];
    for (int i = threadIdx.x; i < n * n * n; i += blockDim.x) {
        const int x = i % n, y = (i / n) % n, z = i / (n * n);
        const T al = L.k.helm ? L.alpha[i] : T(0);
        T v;
        if (first) {
            v = relax_value(L.k, T(0), T(0), L.rhs[i], al);
        } else {
            const long long g = grown_index<T>(n, sx, x, y, z);
            T acc = T(0);
#pragma unroll
            for (int j = 0; j < ShapeLap7::NT; j++) {
                const long long o = ShapeLap7::off(j, 0) + Sy * ShapeLap7::off(j, 1) + Sz * ShapeLap7::off(j, 2);
                acc = dmadd(acc, L.crelax.c[j], src[g + o]);
            }
            v = relax_value(L.k, acc, src[g], L.rhs[i], al);
        }
        store_periodic(dst, n, sx, x, y, z, v);
    }
    __syncthreads();
}
template <typename T>
__device__ void coarse_zero(const CoarseLevel<T>& L, int cur)
{
    const long long m = (long long)L.k.sx * (L.k.n + 2) * (L.k.n + 2);
    for (long long i = threadIdx.x; i < m; i += blockDim.x) L.phi[cur][i] = T(0);
    __syncthreads();
}
// returns the buffer index holding the result
template <typename T>
__device__ int coarse_sweeps(const CoarseLevel<T>& L, int cur, int k, bool zero_start)
{
    for (int s = 0; s < k; s++) {
        coarse_relax(L, cur, zero_start && s == 0);
        cur = 1 - cur;
    }
    if (zero_start && k == 0) coarse_zero(L, cur);
    return cur;
}

// The coarse cycle of one solve, run by one whole CTA; smem is the dynamic shared-memory arena
// (used when ga.in_smem), off the element offsets of each level's buffers in it.
template <typename T>
__device__ void coarse_cycle_body(const CoarseArgs<T>& ga, const CoarseOffsets& off, unsigned char* coarse_smem)
{
    // level descriptors, shared by the block (in shared-memory mode they point into the arena)
    __shared__ CoarseLevel<T> lvs[kMaxCoarse];
    if (threadIdx.x == 0) {
        T* base = reinterpret_cast<T*>(coarse_smem);
        for (int l = 0; l <= ga.top; l++) {
            CoarseLevel<T> L = ga.lv[l];
            if (ga.in_smem) {
                L.phi[0] = base + off.o[l][0];
                L.phi[1] = base + off.o[l][1];
                L.rhs = base + off.o[l][2];
                if (L.k.helm) L.alpha = base + off.o[l][3];
            }
            lvs[l] = L;
        }
    }
    __syncthreads();
    if (ga.in_smem) {
        // rho of the entry level and every alpha come in
        for (int l = 0; l <= ga.top; l++) {
            const int n3 = ga.lv[l].k.n * ga.lv[l].k.n * ga.lv[l].k.n;
            if (l == ga.top)
                for (int i = threadIdx.x; i < n3; i += blockDim.x) lvs[l].rhs[i] = ga.lv[l].rhs[i];
            if (ga.lv[l].k.helm)
                for (int i = threadIdx.x; i < n3; i += blockDim.x) const_cast<T*>(lvs[l].alpha)[i] = ga.lv[l].alpha[i];
        }
        __syncthreads();
    }
    const CoarseArgs<T>& a = ga;
    int cur[kMaxCoarse];
    // down: pre-smoothing from zero, residual restriction
    for (int l = a.top; l > 0; l--) {
        const CoarseLevel<T>& L = lvs[l];
        CoarseLevel<T> const& C = lvs[l - 1];
        cur[l] = coarse_sweeps(L, 0, a.nu1, true);
        const int nf = L.k.n, nc = nf / 2, sx = L.k.sx;
        const long long Sy = sx, Sz = (long long)sx * (nf + 2);
        const T* phi = L.phi[cur[l]];
        for (int i = threadIdx.x; i < nc * nc * nc; i += blockDim.x) {
            const int cx = i % nc, cy = (i / nc) % nc, cz = i / (nc * nc);
            T acc = T(0);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int fx = 2 * cx + (k & 1), fy = 2 * cy + ((k >> 1) & 1), fz = 2 * cz + (k >> 2);
                const int fi = fx + nf * (fy + nf * fz);
                const T al = L.k.helm ? L.alpha[fi] : T(0);
                const T r = fine_residual(phi, grown_index<T>(nf, sx, fx, fy, fz), Sy, Sz, L.rhs[fi], al, L.k.helm,
                                          L.cres, a.beta);
                acc = dmadd(acc, T(1.0 / 8), r);
            }
            C.rhs[i] = acc;
        }
        __syncthreads();
    }
    // bottom
    {
        const CoarseLevel<T>& B = lvs[0];
        if (a.direct) {
            const int n = B.k.n, N = n * n * n;
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                T acc = T(0);
                for (int j = 0; j < N; j++) acc = dmadd(acc, a.ainv[(long long)i * N + j], B.rhs[j]);
                store_periodic(B.phi[0], n, B.k.sx, i % n, (i / n) % n, i / (n * n), acc);
            }
            __syncthreads();
            cur[0] = 0;
        } else {
            cur[0] = coarse_sweeps(B, 0, a.nu_bottom, true);
        }
    }
    // up: prolongation, post-smoothing
    for (int l = 1; l <= a.top; l++) {
        const CoarseLevel<T>& L = lvs[l];
        const CoarseLevel<T>& C = lvs[l - 1];
        const int nf = L.k.n, nc = nf / 2;
        T* phi = L.phi[cur[l]];
        const T* d = C.phi[cur[l - 1]];
        for (int i = threadIdx.x; i < nf * nf * nf; i += blockDim.x) {
            const int x = i % nf, y = (i / nf) % nf, z = i / (nf * nf);
            const T dv = d[grown_index<T>(nc, C.k.sx, x / 2, y / 2, z / 2)];
            const long long g = grown_index<T>(nf, L.k.sx, x, y, z);
            store_periodic(phi, nf, L.k.sx, x, y, z, dadd(phi[g], dmul(T(1), dv)));
        }
        __syncthreads();
        cur[l] = coarse_sweeps(L, cur[l], a.nu2, false);
    }
    // leave the result in buffer 0 of the top level (in global memory)
    if (a.in_smem || cur[a.top] == 1) {
        const CoarseLevel<T>& L = lvs[a.top];
        const long long m = (long long)L.k.sx * (L.k.n + 2) * (L.k.n + 2);
        const T* src = L.phi[cur[a.top]];
        for (long long i = threadIdx.x; i < m; i += blockDim.x) ga.lv[a.top].phi[0][i] = src[i];
    }
    __syncthreads();   // the descriptor table may be reused by the next solve of this block
}

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse_cycle(const CoarseArgs<T> ga, const CoarseOffsets off)
{
    extern __shared__ __align__(16) unsigned char coarse_smem[];
    coarse_cycle_body(ga, off, coarse_smem);
}

// One CTA per solve of a batch; *count solves are live (the grid is sized for the largest batch).
template <typename T>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse_cycle_batch(const CoarseArgs<T>* __restrict__ args,
                                                                       const CoarseOffsets* __restrict__ offs,
                                                                       const int* __restrict__ count)
{
    extern __shared__ __align__(16) unsigned char coarse_smem[];
    const int n = *count;
    for (int b = blockIdx.x; b < n; b += gridDim.x) coarse_cycle_body(args[b], offs[b], coarse_smem);
}

// ---- host helpers shared by the solvers -----------------------------------------------------------
// 7-point coefficients times s (the reference's Stencil * scale: coefficient*s unless s == 1)
template <typename T>
static inline Coefs<T> lap7_coefs(double s)
{
    Coefs<T> cf;
    for (int j = 0; j < 13; j++) cf.c[j] = T(0);
    for (int j = 0; j < 7; j++) {
        const double c = (j == 0) ? -6.0 : 1.0;
        cf.c[j] = (T)((s != 1.0) ? c * s : c);
    }
    return cf;
}

// Jacobi weight lambda = omega*h^2/6 of the Poisson form
static inline double mg_lambda(double omega, double h) { return (omega * (h * h)) / 6.0; }

} // namespace pb
