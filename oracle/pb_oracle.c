/*
 * CPU restatement ("port") of the reference's structured-grid hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg compare the CUDA library against. Nothing on the product path links or calls
 * it. It is pinned against the reference itself (oracle/_ref/libproto_ref.so, built from the
 * reference headers by oracle/build_oracle.py) and against the committed fixtures in tests/golden/.
 *
 * Floating-point operation order follows the reference CPU path exactly (compile with
 * -ffp-contract=off), so results are bitwise equal to it:
 *   - Stencil::hostApply (include/base/implem/Proto_StencilImplem.H:725-828): destination zeroed
 *     for "|=", coefficients pre-multiplied by the scale when scale != 1, then for each term in
 *     insertion order dst += coef*src.
 *   - BoxData algebra / forall bodies: one rounding per written operator, left to right.
 *   - Reduction<T,OP,HOST>::update (include/base/implem/Proto_ReductionImplem.H:62-101),
 *     including Max's initial value numeric_limits<double>::min().
 * Layout: a field on box [lo,hi] is stored x fastest, index = Box::sindex
 * (include/base/implem/Proto_BoxImplem.H:76-86); components are contiguous blocks of box size.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { int lo[3], hi[3]; } obox;

static inline long bsize(const obox* b, int d) { return (long)b->hi[d] - b->lo[d] + 1; }
static inline long bvol(const obox* b)
{
    if (b->hi[0] < b->lo[0] || b->hi[1] < b->lo[1] || b->hi[2] < b->lo[2]) return 0;
    return bsize(b, 0) * bsize(b, 1) * bsize(b, 2);
}
static inline int bempty(const obox* b) { return bvol(b) == 0; }
/* Box::sindex: x-fastest linear index of p within [lo,hi] (unsigned 32-bit in the reference). */
static inline long sindex(const int* p, const obox* b)
{
    return (long)(p[0] - b->lo[0]) + bsize(b, 0) * ((long)(p[1] - b->lo[1]) + bsize(b, 1) * (long)(p[2] - b->lo[2]));
}
static inline int contains(const obox* b, const int* p)
{
    for (int d = 0; d < 3; d++) if (p[d] < b->lo[d] || p[d] > b->hi[d]) return 0;
    return 1;
}
static obox intersect(const obox* a, const obox* b)
{
    obox r;
    for (int d = 0; d < 3; d++) {
        r.lo[d] = a->lo[d] > b->lo[d] ? a->lo[d] : b->lo[d];
        r.hi[d] = a->hi[d] < b->hi[d] ? a->hi[d] : b->hi[d];
    }
    return r;
}

/* ---------------------------------------------------------------------------------------------
 * Box index-space transforms (include/base/implem/Proto_BoxImplem.H:506-564)
 * ------------------------------------------------------------------------------------------- */
static int coarsen_lo(int v, int r) { return v < 0 ? ((-v) % r == 0 ? -((-v) / r) : -((-v) / r + 1)) : v / r; }
static int coarsen_hi(int v, int r) { return v < 0 ? (v % r == 0 ? -((-v) / r) : -((-v) / r + 1)) : v / r; }

void or_box_coarsen(const int* lo, const int* hi, const int* r, int* olo, int* ohi)
{
    for (int d = 0; d < 3; d++) { olo[d] = coarsen_lo(lo[d], r[d]); ohi[d] = coarsen_hi(hi[d], r[d]); }
}

/* taperCoarsen: high = Point division (rounds toward -infinity, Proto_PointImplem.H:212-239),
 * low = ceil(lo / r) */
void or_box_taper_coarsen(const int* lo, const int* hi, const int* r, int* olo, int* ohi)
{
    for (int d = 0; d < 3; d++) {
        ohi[d] = coarsen_hi(hi[d], r[d]);
        olo[d] = (int)ceil((double)lo[d] / (double)r[d]);
    }
}

/* ---------------------------------------------------------------------------------------------
 * Stencil apply (Stencil::hostApply order). Index box 'ib' in the stencil's index space:
 * destination point = p*dstRatio + dstShift, source point = p*srcRatio + offset.
 * A pencil (fixed y,z) whose first destination point lies outside the destination box is skipped,
 * as in the reference; the caller guarantees the remaining points of kept pencils are inside.
 * ------------------------------------------------------------------------------------------- */
int or_stencil_apply(const double* coefs, const int* offs, int n, const int* meta,
                     const double* src, const int* srcLo, const int* srcHi,
                     double* dst, const int* dstLo, const int* dstHi,
                     const int* boxLo, const int* boxHi, int initToZero, double scale, int ncomp)
{
    obox sb, db, ib;
    memcpy(sb.lo, srcLo, 12); memcpy(sb.hi, srcHi, 12);
    memcpy(db.lo, dstLo, 12); memcpy(db.hi, dstHi, 12);
    memcpy(ib.lo, boxLo, 12); memcpy(ib.hi, boxHi, 12);
    if (bempty(&ib) || n == 0) return 0;
    const int* sr = meta; const int* dr = meta + 3; const int* ds = meta + 6;
    long svol = bvol(&sb), dvol = bvol(&db);
    double* c = (double*)malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) c[j] = (scale != 1.0) ? coefs[j] * scale : coefs[j];
    long nx = bsize(&ib, 0), ny = bsize(&ib, 1), nz = bsize(&ib, 2);
    for (int comp = 0; comp < ncomp; comp++) {
        const double* s = src + comp * svol;
        double* o = dst + comp * dvol;
        #pragma omp parallel for collapse(2) schedule(static)
        for (long k = 0; k < nz; k++)
        for (long jy = 0; jy < ny; jy++) {
            int p0[3] = {ib.lo[0], ib.lo[1] + (int)jy, ib.lo[2] + (int)k};
            int d0[3] = {p0[0]*dr[0] + ds[0], p0[1]*dr[1] + ds[1], p0[2]*dr[2] + ds[2]};
            if (!contains(&db, d0)) continue;
            for (long i = 0; i < nx; i++) {
                int p[3] = {p0[0] + (int)i, p0[1], p0[2]};
                int dp[3] = {p[0]*dr[0] + ds[0], d0[1], d0[2]};
                long di = sindex(dp, &db);
                double acc = initToZero ? 0.0 : o[di];
                if (scale != 0.0) {
                    for (int j = 0; j < n; j++) {
                        int sp[3] = {p[0]*sr[0] + offs[3*j], p[1]*sr[1] + offs[3*j+1], p[2]*sr[2] + offs[3*j+2]};
                        acc = acc + c[j] * s[sindex(sp, &sb)];
                    }
                }
                o[di] = acc;
            }
        }
    }
    free(c);
    return 0;
}

/* Box inference of Stencil::apply for an empty box: indexDomain(dst) & indexRange(src)
 * (include/base/implem/Proto_StencilImplem.H:324-346, 412-431). span = bounding box of offsets. */
void or_stencil_infer_box(const int* offs, int n, const int* meta, const int* srcLo, const int* srcHi,
                          const int* dstLo, const int* dstHi, int* outLo, int* outHi)
{
    int spLo[3] = {0, 0, 0}, spHi[3] = {0, 0, 0};
    for (int j = 0; j < n; j++)
        for (int d = 0; d < 3; d++) {
            int v = offs[3*j+d];
            if (j == 0 || v < spLo[d]) spLo[d] = v;
            if (j == 0 || v > spHi[d]) spHi[d] = v;
        }
    int rLo[3], rHi[3], dLo[3], dHi[3], t1[3], t2[3];
    for (int d = 0; d < 3; d++) { t1[d] = srcLo[d] - spLo[d]; t2[d] = srcHi[d] - spHi[d]; }
    or_box_taper_coarsen(t1, t2, meta, rLo, rHi);
    for (int d = 0; d < 3; d++) { t1[d] = dstLo[d] - meta[6+d]; t2[d] = dstHi[d] - meta[6+d]; }
    or_box_taper_coarsen(t1, t2, meta + 3, dLo, dHi);
    for (int d = 0; d < 3; d++) {
        outLo[d] = rLo[d] > dLo[d] ? rLo[d] : dLo[d];
        outHi[d] = rHi[d] < dHi[d] ? rHi[d] : dHi[d];
    }
}

/* ---------------------------------------------------------------------------------------------
 * Piecewise-constant prolongation (InterpStencil::Constant, include/base/implem/
 * Proto_InterpStencilDefs.H:1-15 applied through InterpStencil::apply, Proto_InterpStencilImplem.H:91-118).
 * Every coefficient is 1.0 and every stage starts from zero, so the composite is
 * dst = src(p / r) ("|=") or dst = dst + src(p / r) ("+="), scaled by 'scale' when scale != 1.
 * ------------------------------------------------------------------------------------------- */
int or_interp_constant(int r, const double* src, const int* srcLo, const int* srcHi,
                       double* dst, const int* dstLo, const int* dstHi, int overwrite, double scale)
{
    obox sb, db;
    memcpy(sb.lo, srcLo, 12); memcpy(sb.hi, srcHi, 12);
    memcpy(db.lo, dstLo, 12); memcpy(db.hi, dstHi, 12);
    /* range(src) & dst */
    obox rb;
    for (int d = 0; d < 3; d++) { rb.lo[d] = sb.lo[d]*r; rb.hi[d] = sb.hi[d]*r + r - 1; }
    rb = intersect(&rb, &db);
    if (bempty(&rb)) return 0;
    double coef = scale;   /* (scale * 1.0) */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = rb.lo[2]; z <= rb.hi[2]; z++)
    for (int y = rb.lo[1]; y <= rb.hi[1]; y++)
    for (int x = rb.lo[0]; x <= rb.hi[0]; x++) {
        int p[3] = {x, y, z};
        int c[3] = {coarsen_lo(x, r), coarsen_lo(y, r), coarsen_lo(z, r)};
        double v = src[sindex(c, &sb)];
        long di = sindex(p, &db);
        double acc = overwrite ? 0.0 : dst[di];
        dst[di] = acc + coef * v;
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Ghost exchange. For a layout of disjoint patches tiling 'domain', a ghost cell of a patch takes
 * the value of the valid cell at its periodic image (the unique result of
 * LevelBoxData::exchange, include/base/implem/Proto_LevelBoxDataImplem.H:315-329,900-951).
 * Cells outside the domain in a non-periodic direction are left untouched.
 * patches: npatch boxes (lo,hi interleaved as 6 ints); data[i] points at patch i's grown box.
 * ------------------------------------------------------------------------------------------- */
int or_exchange(int npatch, const int* boxes, const int* ghost, const int* domLo, const int* domHi,
                const int* periodic, double** data, int ncomp)
{
    obox dom;
    memcpy(dom.lo, domLo, 12); memcpy(dom.hi, domHi, 12);
    long L[3] = {bsize(&dom, 0), bsize(&dom, 1), bsize(&dom, 2)};
    for (int i = 0; i < npatch; i++) {
        obox vb, gb;
        memcpy(vb.lo, boxes + 6*i, 12); memcpy(vb.hi, boxes + 6*i + 3, 12);
        for (int d = 0; d < 3; d++) { gb.lo[d] = vb.lo[d] - ghost[d]; gb.hi[d] = vb.hi[d] + ghost[d]; }
        long gvol = bvol(&gb);
        #pragma omp parallel for collapse(2) schedule(static)
        for (int z = gb.lo[2]; z <= gb.hi[2]; z++)
        for (int y = gb.lo[1]; y <= gb.hi[1]; y++)
        for (int x = gb.lo[0]; x <= gb.hi[0]; x++) {
            int p[3] = {x, y, z};
            if (contains(&vb, p)) continue;
            int q[3];
            int skip = 0;
            for (int d = 0; d < 3; d++) {
                q[d] = p[d];
                if (q[d] < dom.lo[d] || q[d] > dom.hi[d]) {
                    if (!periodic[d]) { skip = 1; break; }
                    long t = ((long)q[d] - dom.lo[d]) % L[d];
                    if (t < 0) t += L[d];
                    q[d] = (int)(t + dom.lo[d]);
                }
            }
            if (skip) continue;
            for (int j = 0; j < npatch; j++) {
                obox vj, gj;
                memcpy(vj.lo, boxes + 6*j, 12); memcpy(vj.hi, boxes + 6*j + 3, 12);
                if (!contains(&vj, q)) continue;
                for (int d = 0; d < 3; d++) { gj.lo[d] = vj.lo[d] - ghost[d]; gj.hi[d] = vj.hi[d] + ghost[d]; }
                long gjvol = bvol(&gj);
                for (int c = 0; c < ncomp; c++)
                    data[i][c*gvol + sindex(p, &gb)] = data[j][c*gjvol + sindex(q, &gj)];
                break;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Reductions (Reduction<T,OP,HOST>): op 0 Max, 1 Min, 2 Abs, 3 Sum, 4 SumAbs, 5 SumSquare.
 * Host order is sequential; max/min/abs are order independent.
 * ------------------------------------------------------------------------------------------- */
static inline double rmax(double a, double b) { return (a < b) ? b : a; }   /* std::max */
static inline double rmin(double a, double b) { return (b < a) ? b : a; }   /* std::min */
static inline double upd_abs(double v1, double v2) { return v2 > 0 ? rmax(v1, v2) : rmax(v1, -v2); }

double or_reduce(int op, const double* d, long n)
{
    double v;
    switch (op) {
        case 0: v = DBL_MIN; for (long i = 0; i < n; i++) v = rmax(v, d[i]); return v;
        case 1: v = DBL_MAX; for (long i = 0; i < n; i++) v = rmin(v, d[i]); return v;
        case 2: v = 0.0; for (long i = 0; i < n; i++) v = upd_abs(v, d[i]); return v;
        case 3: v = 0.0; for (long i = 0; i < n; i++) v += d[i]; return v;
        case 4: v = 0.0; for (long i = 0; i < n; i++) v += (d[i] > 0 ? d[i] : -d[i]); return v;
        case 5: v = 0.0; for (long i = 0; i < n; i++) v += d[i] * d[i]; return v;
    }
    return 0.0;
}

/* absMax over the valid box of a grown single-box field, in parallel (order independent) */
static double absmax_valid(const double* u, int N, int g)
{
    long S = N + 2*g;
    double best = 0.0;
    #pragma omp parallel for reduction(max:best) schedule(static)
    for (int z = 0; z < N; z++) {
        double b = 0.0;
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) b = upd_abs(b, u[(x+g) + S*((y+g) + S*(long)(z+g))]);
        if (b > best) best = b;
    }
    return best;
}

/* ---------------------------------------------------------------------------------------------
 * Single-box periodic levels. A level of edge N with ghost width g is an (N+2g)^3 array, x fastest.
 * ------------------------------------------------------------------------------------------- */
#define IDX(x, y, z, S) ((long)(x) + (long)(S) * ((long)(y) + (long)(S) * (long)(z)))

static void fill_periodic(double* u, int N, int g)
{
    long S = N + 2*g;
    #pragma omp parallel for schedule(static)
    for (int z = 0; z < S; z++)
        for (int y = 0; y < S; y++)
            for (int x = 0; x < S; x++) {
                if (x >= g && x < N+g && y >= g && y < N+g && z >= g && z < N+g) continue;
                int qx = ((x - g) % N + N) % N + g, qy = ((y - g) % N + N) % N + g, qz = ((z - g) % N + N) % N + g;
                u[IDX(x, y, z, S)] = u[IDX(qx, qy, qz, S)];
            }
}

/* 7-point Laplacian in Stencil::Laplacian insertion order: 0, +x, -x, +y, -y, +z, -z
 * (include/base/implem/Proto_StencilDefs.H:77-87) */
static const int LAP7_OFF[7][3] = {{0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
static const double LAP7_C[7] = {-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};

static inline double lap7(const double* u, long i, long S, const double* c, double acc)
{
    for (int j = 0; j < 7; j++)
        acc = acc + c[j] * u[i + LAP7_OFF[j][0] + S * (LAP7_OFF[j][1] + S * LAP7_OFF[j][2])];
    return acc;
}
static void scaled(const double* c0, int n, double s, double* c) { for (int j = 0; j < n; j++) c[j] = (s != 1.0) ? c0[j]*s : c0[j]; }

typedef struct {
    int N;                 /* finest edge */
    int levels;            /* finest level index; levels+1 grids, edge N >> (levels - l) */
    int nu1, nu2, nuBottom;
    double omega, beta;
    int helm;              /* 0: Poisson form (L phi = rho), 1: Helmholtz form (alpha*phi - beta*L phi = f) */
    double** phi;          /* per level (index l, finest = levels): (n+2)^3 */
    double** rhs;          /* per level: n^3 */
    double** alpha;        /* per level: n^3 (Helmholtz) */
    double** tmp;          /* per level: n^3 */
    int bottom;            /* 0: nuBottom sweeps on the coarsest grid, 1: exact solve with ainv */
    double* ainv;          /* bottom == 1: inverse of the coarsest operator */
} or_cs;

static int lvl_n(const or_cs* m, int l) { return m->N >> (m->levels - l); }
static double lvl_h(const or_cs* m, int l) { return (double)(1 << (m->levels - l)) / (double)m->N; }

/* residual r = rho + L(phi, -1/h^2) (Poisson) or f - (alpha*phi - beta*L(phi, 1/h^2)) (Helmholtz) */
static void cs_residual(const or_cs* m, int l, double* r)
{
    int n = lvl_n(m, l); long S = n + 2;
    double h = lvl_h(m, l), hsqinv = 1. / (h * h);
    const double* u = m->phi[l]; const double* f = m->rhs[l];
    double c[7];
    if (!m->helm) scaled(LAP7_C, 7, -hsqinv, c); else scaled(LAP7_C, 7, hsqinv, c);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
        long i = IDX(x+1, y+1, z+1, S), o = IDX(x, y, z, n);
        if (!m->helm) {
            r[o] = lap7(u, i, S, c, 0.0 + f[o]);
        } else {
            double lp = lap7(u, i, S, c, 0.0);
            r[o] = f[o] - (m->alpha[l][o] * u[i] - m->beta * lp);
        }
    }
}

static void cs_relax(or_cs* m, int l, int sweeps)
{
    int n = lvl_n(m, l); long S = n + 2;
    double h = lvl_h(m, l), hsqinv = 1. / (h * h);
    double w = m->omega / 6.0, lambda = (m->omega * (h * h)) / 6.0;
    double diagB = 6.0 * m->beta * hsqinv;
    double cw[7]; scaled(LAP7_C, 7, w, cw);
    double* u = m->phi[l]; double* t = m->tmp[l]; const double* f = m->rhs[l];
    for (int s = 0; s < sweeps; s++) {
        fill_periodic(u, n, 1);
        if (!m->helm) {
            #pragma omp parallel for collapse(2) schedule(static)
            for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
                long o = IDX(x, y, z, n);
                double tv = lap7(u, IDX(x+1, y+1, z+1, S), S, cw, 0.0);
                t[o] = tv + (-lambda) * f[o];
            }
        } else {
            cs_residual(m, l, t);
            #pragma omp parallel for collapse(2) schedule(static)
            for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
                long o = IDX(x, y, z, n);
                t[o] = (m->omega * t[o]) / (m->alpha[l][o] + diagB);
            }
        }
        #pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
            long i = IDX(x+1, y+1, z+1, S);
            u[i] = u[i] + t[IDX(x, y, z, n)];
        }
    }
}

/* AvgDown(2): 8 fine cells in Box([0,1]^3) iteration order (x fastest), coefficient 1/8 each */
static void avgdown(const double* fine, int nf, double* crse)
{
    int nc = nf / 2;
    const double c = 1.0 / 8;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nc; z++) for (int y = 0; y < nc; y++) for (int x = 0; x < nc; x++) {
        double acc = 0.0;
        for (int kz = 0; kz < 2; kz++) for (int ky = 0; ky < 2; ky++) for (int kx = 0; kx < 2; kx++)
            acc = acc + c * fine[IDX(2*x+kx, 2*y+ky, 2*z+kz, nf)];
        crse[IDX(x, y, z, nc)] = acc;
    }
}

static double cs_resnorm(or_cs* m, int l)
{
    int n = lvl_n(m, l); long S = n + 2;
    double h = lvl_h(m, l), hsqinv = 1. / (h * h);
    double* u = m->phi[l];
    fill_periodic(u, n, 1);
    if (m->helm) {
        cs_residual(m, l, m->tmp[l]);
        return or_reduce(2, m->tmp[l], (long)n*n*n);
    }
    double c[7]; scaled(LAP7_C, 7, hsqinv, c);
    const double* f = m->rhs[l];
    double best = 0.0;
    #pragma omp parallel for reduction(max:best) schedule(static)
    for (int z = 0; z < n; z++) {
        double b = 0.0;
        for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
            long o = IDX(x, y, z, n);
            b = upd_abs(b, lap7(u, IDX(x+1, y+1, z+1, S), S, c, 0.0 - f[o]));
        }
        if (b > best) best = b;
    }
    return best;
}

/* Exact coarsest solve (no counterpart in the reference, whose bottom solver is relaxation): the
 * inverse of the coarsest operator by Gauss-Jordan elimination with partial pivoting on [A | I].
 * A = L(., 1/h^2) (Poisson form) or diag(alpha) - beta*L(., 1/h^2) (Helmholtz form), periodic;
 * a singular A (Poisson, or alpha == 0 everywhere) gets (6/h^2)/N added to every entry. Each row
 * takes alpha first, then the 7-point terms in insertion order. Returns 0 on success. */
static int cs_coarse_inverse(int n0, double h, int helm, double beta, const double* alpha, double* inv)
{
    int N = n0 * n0 * n0;
    double hs = 1. / (h * h);
    long W = 2L * N;
    double* M = (double*)calloc((size_t)N * W, sizeof(double));
    int singular = !helm;
    if (helm) {
        singular = 1;
        for (int i = 0; i < N; i++) singular = singular && alpha[i] == 0.0;
    }
    for (int z = 0; z < n0; z++) for (int y = 0; y < n0; y++) for (int x = 0; x < n0; x++) {
        int i = x + n0 * (y + n0 * z);
        if (helm) M[i * W + i] += alpha[i];
        for (int j = 0; j < 7; j++) {
            int qx = (x + LAP7_OFF[j][0] + n0) % n0, qy = (y + LAP7_OFF[j][1] + n0) % n0, qz = (z + LAP7_OFF[j][2] + n0) % n0;
            int k = qx + n0 * (qy + n0 * qz);
            double t = helm ? (-beta) * (LAP7_C[j] * hs) : (LAP7_C[j] * hs);
            M[i * W + k] += t;
        }
    }
    if (singular) {
        double reg = (6.0 * hs) / N;
        for (int i = 0; i < N; i++) for (int k = 0; k < N; k++) M[i * W + k] += reg;
    }
    for (int i = 0; i < N; i++) M[i * W + N + i] = 1.0;
    for (int c = 0; c < N; c++) {
        int p = c;
        double best = fabs(M[c * W + c]);
        for (int r = c + 1; r < N; r++)
            if (fabs(M[r * W + c]) > best) { best = fabs(M[r * W + c]); p = r; }
        if (best == 0.0) { free(M); return -1; }
        if (p != c)
            for (long j = 0; j < W; j++) { double t = M[p * W + j]; M[p * W + j] = M[c * W + j]; M[c * W + j] = t; }
        double piv = M[c * W + c];
        for (long j = 0; j < W; j++) M[c * W + j] = M[c * W + j] / piv;
        for (int r = 0; r < N; r++) {
            if (r == c) continue;
            double f = M[r * W + c];
            if (f != 0.0)
                for (long j = 0; j < W; j++) M[r * W + j] = M[r * W + j] - f * M[c * W + j];
        }
    }
    for (int i = 0; i < N; i++) for (int k = 0; k < N; k++) inv[(long)i * N + k] = M[i * W + N + k];
    free(M);
    return 0;
}

/* phi = Ainv * rhs on the coarsest level, products summed in column order */
static void cs_bottom_direct(or_cs* m)
{
    int n = lvl_n(m, 0), N = n * n * n;
    long S = n + 2;
    for (int i = 0; i < N; i++) {
        double acc = 0.0;
        for (int j = 0; j < N; j++) acc = acc + m->ainv[(long)i * N + j] * m->rhs[0][j];
        int x = i % n, y = (i / n) % n, z = i / (n * n);
        m->phi[0][IDX(x + 1, y + 1, z + 1, S)] = acc;
    }
    fill_periodic(m->phi[0], n, 1);
}

static void cs_vcycle(or_cs* m, int l)
{
    if (l > 0) {
        int n = lvl_n(m, l), nc = n / 2;
        cs_relax(m, l, m->nu1);
        fill_periodic(m->phi[l], n, 1);
        cs_residual(m, l, m->tmp[l]);
        avgdown(m->tmp[l], n, m->rhs[l-1]);
        memset(m->phi[l-1], 0, sizeof(double) * (size_t)(nc+2)*(nc+2)*(nc+2));
        cs_vcycle(m, l - 1);
        long S = n + 2, Sc = nc + 2;
        double* u = m->phi[l]; const double* d = m->phi[l-1];
        #pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
            long i = IDX(x+1, y+1, z+1, S);
            u[i] = u[i] + 1.0 * d[IDX(x/2+1, y/2+1, z/2+1, Sc)];
        }
        cs_relax(m, l, m->nu2);
    } else if (m->bottom) {
        cs_bottom_direct(m);
    } else {
        cs_relax(m, l, m->nuBottom);
    }
}

/* Correction-scheme multigrid on one periodic N^3 box per level; same arithmetic as the
 * reference's archived LevelMultigrid (examples/_archived/LevelMultigrid/src/LevelMultigrid.cpp:
 * pointRelax 90-114, coarseResidual 48-69, resnorm 71-88, fineInterp 116-131, vCycle 133-158) with
 * the smoother weight omega/6 (the archived solver is omega = 1/2) and the sweep counts as
 * parameters, plus the Helmholtz form. rhs/phi: N^3 (x fastest). hist: maxIter+1 entries.
 * Returns the number of V-cycles run. */
int or_mg_cs(int N, int levels, int nu1, int nu2, int nuBottom, double omega, double beta,
             const double* alpha, int maxIter, double tol, const double* rhs, double* phi, double* hist,
             int bottom)
{
    or_cs m;
    m.N = N; m.levels = levels; m.nu1 = nu1; m.nu2 = nu2; m.nuBottom = nuBottom;
    m.omega = omega; m.beta = beta; m.helm = alpha != 0;
    int nl = levels + 1;
    m.phi = (double**)calloc(nl, sizeof(double*));
    m.rhs = (double**)calloc(nl, sizeof(double*));
    m.alpha = (double**)calloc(nl, sizeof(double*));
    m.tmp = (double**)calloc(nl, sizeof(double*));
    for (int l = 0; l < nl; l++) {
        long n = lvl_n(&m, l);
        m.phi[l] = (double*)calloc((size_t)(n+2)*(n+2)*(n+2), sizeof(double));
        m.rhs[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
        m.alpha[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
        m.tmp[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
    }
    long S = N + 2;
    for (int z = 0; z < N; z++) for (int y = 0; y < N; y++) for (int x = 0; x < N; x++) {
        m.phi[levels][IDX(x+1, y+1, z+1, S)] = phi[IDX(x, y, z, N)];
        m.rhs[levels][IDX(x, y, z, N)] = rhs[IDX(x, y, z, N)];
    }
    if (alpha) {
        memcpy(m.alpha[levels], alpha, sizeof(double) * (size_t)N*N*N);
        for (int l = levels; l > 0; l--) avgdown(m.alpha[l], lvl_n(&m, l), m.alpha[l-1]);
    }
    m.bottom = bottom;
    m.ainv = 0;
    if (bottom) {
        long n0 = lvl_n(&m, 0), N0 = n0 * n0 * n0;
        m.ainv = (double*)calloc((size_t)(N0 * N0), sizeof(double));
        if (cs_coarse_inverse((int)n0, lvl_h(&m, 0), m.helm, beta, m.alpha[0], m.ainv) != 0) { free(m.ainv); return -1; }
    }
    double r0 = cs_resnorm(&m, levels);
    hist[0] = r0;
    int it = 0;
    while (it < maxIter) {
        cs_vcycle(&m, levels);
        double r = cs_resnorm(&m, levels);
        hist[++it] = r;
        if (r < tol * r0) break;
    }
    for (int z = 0; z < N; z++) for (int y = 0; y < N; y++) for (int x = 0; x < N; x++)
        phi[IDX(x, y, z, N)] = m.phi[levels][IDX(x+1, y+1, z+1, S)];
    for (int l = 0; l < nl; l++) { free(m.phi[l]); free(m.rhs[l]); free(m.alpha[l]); free(m.tmp[l]); }
    free(m.phi); free(m.rhs); free(m.alpha); free(m.tmp);
    free(m.ainv);
    return it;
}

/* ---------------------------------------------------------------------------------------------
 * FAS multigrid with the 4th-order flux-form Laplacian: LevelMultigridSolver<BoxOp_Laplace>
 * (include/utils/implem/Proto_LevelMultigridSolverImplem.H:85-433; BoxOp::operator(),
 * include/base/implem/Proto_BoxOpImplem.H:125-172; BoxOp_Laplace::flux,
 * examples/_common/BoxOp_Laplace.H:22-27) on one periodic box per level, ghost width 2.
 *   flux_d(q)  = sum_k g_k u[q + k e_d], k = -2,-1,0,1 (DiffCellToFace(d, Lo, 4) * 1/dx, |=)
 *   div(p)     = 0; per d: div += c+ * flux_d(p + e_d); div += c0 * flux_d(p)   (DIV * 1/dx, +=)
 *   op(p)      = (0 + div) * (-1)                                             (fluxScale = -1)
 *   relax      : res = op(u) + f;  u += (-lambda) * res, lambda = 0.5 / (6/dx^2)
 *   coarse force: AvgDown(op(u) + f) - op_c(AvgDown(u));  correction: u += 1.0 * (-(c0 - c))
 * V(6,6), 10 bottom sweeps. Per-patch evaluation in the reference equals this per-cell evaluation
 * (each cell's operations depend only on values, and ghosts hold the periodic images).
 * ------------------------------------------------------------------------------------------- */
static void fas_op(const double* u, int n, double dx, const double* dc, double* out)
{
    /* dc: 4 face-gradient coefficients then the 2 divergence coefficients (term order +e, 0) */
    long S = n + 4;
    double g[4], cp = dc[4], c0 = dc[5];
    for (int k = 0; k < 4; k++) g[k] = dc[k];
    (void)dx;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
        long i = IDX(x+2, y+2, z+2, S);
        double div = 0.0;
        for (int d = 0; d < 3; d++) {
            long e = d == 0 ? 1 : (d == 1 ? S : S*S);
            double fp = 0.0, fm = 0.0;
            for (int k = 0; k < 4; k++) fp = fp + g[k] * u[i + e + (k - 2) * e];
            for (int k = 0; k < 4; k++) fm = fm + g[k] * u[i + (k - 2) * e];
            div = div + cp * fp;
            div = div + c0 * fm;
        }
        out[IDX(x, y, z, n)] = (0.0 + div) * -1.0;
    }
}

/* the operator's coefficients at spacing dx: DiffCellToFace(.,Lo,4) = {1,-15,15,-1} * (1/12),
 * folded by 1/dx; divergence 1.0*Shift(+e) - 1.0*Shift(0), folded by 1/dx */
static void fas_coefs(double dx, double* dc)
{
    const double base[4] = {1.0, -15.0, 15.0, -1.0};
    double s = 1.0 / dx;
    for (int k = 0; k < 4; k++) {
        double c = base[k] * (1.0 / 12.0);
        dc[k] = (s != 1.0) ? c * s : c;
    }
    dc[4] = (s != 1.0) ? 1.0 * s : 1.0;
    dc[5] = (s != 1.0) ? -1.0 * s : -1.0;
}

/* BoxOp<BoxOp_Laplace>::operator()(out, state, scale) on a box (BoxOp::operator(),
 * include/base/implem/Proto_BoxOpImplem.H:130-175; flux: examples/_common/BoxOp_Laplace.H:22-27):
 * divFlux = 0, then per direction divFlux += DIV_d(flux_d, 1/dx) with flux_d |= GRAD_d(state, 1/dx);
 * out = 0 + divFlux; out *= fluxScale; out *= scale when scale != 1. state on [sLo,sHi], out on
 * [oLo,oHi], evaluated on range [rLo,rHi]. */
int or_boxop_laplace(const double* u, const int* sLo, const int* sHi, double* out, const int* oLo, const int* oHi,
                     const int* rLo, const int* rHi, double dx, double fluxScale, double scale)
{
    double dc[6];
    fas_coefs(dx, dc);
    long Sx = (long)sHi[0] - sLo[0] + 1, Sxy = Sx * ((long)sHi[1] - sLo[1] + 1);
    long Ox = (long)oHi[0] - oLo[0] + 1, Oxy = Ox * ((long)oHi[1] - oLo[1] + 1);
    for (int z = rLo[2]; z <= rHi[2]; z++)
        for (int y = rLo[1]; y <= rHi[1]; y++)
            for (int x = rLo[0]; x <= rHi[0]; x++) {
                long c = (x - sLo[0]) + Sx * (y - sLo[1]) + Sxy * (z - sLo[2]);
                double div = 0.0;
                for (int d = 0; d < 3; d++) {
                    long e = d == 0 ? 1 : (d == 1 ? Sx : Sxy);
                    double fp = 0.0, fm = 0.0;
                    for (int k = 0; k < 4; k++) fp = fp + dc[k] * u[c + e + (k - 2) * e];
                    for (int k = 0; k < 4; k++) fm = fm + dc[k] * u[c + (k - 2) * e];
                    div = div + dc[4] * fp;
                    div = div + dc[5] * fm;
                }
                double v = (0.0 + div) * fluxScale;
                if (scale != 1.0) v = v * scale;
                out[(x - oLo[0]) + Ox * (y - oLo[1]) + Oxy * (z - oLo[2])] = v;
            }
    return 0;
}

typedef struct {
    int N, levels;      /* finest edge; number of levels (finest index levels-1) */
    double** u;         /* per level (n+4)^3 */
    double** f;         /* per level n^3 */
    double** c0;        /* per level n^3 (copy of the averaged-down state) */
    double** t;         /* per level n^3 scratch */
    double** r;         /* per level n^3 scratch */
} or_fas;

static int fas_n(const or_fas* m, int l) { return m->N >> (m->levels - 1 - l); }
static double fas_dx(const or_fas* m, int l) { return (double)(1 << (m->levels - 1 - l)) / (double)m->N; }

static void fas_relax(or_fas* m, int l, int sweeps)
{
    int n = fas_n(m, l); long S = n + 4;
    double dx = fas_dx(m, l), dc[6];
    fas_coefs(dx, dc);
    double lambda = 0.5 / ((2.0 * 3) / pow(dx, 2));
    for (int s = 0; s < sweeps; s++) {
        fill_periodic(m->u[l], n, 2);
        fas_op(m->u[l], n, dx, dc, m->t[l]);
        #pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
            long o = IDX(x, y, z, n), i = IDX(x+2, y+2, z+2, S);
            double res = m->t[l][o] + m->f[l][o];
            m->u[l][i] = m->u[l][i] + (-lambda) * res;
        }
    }
}

static void fas_vcycle(or_fas* m, int l)
{
    if (l == 0) { fas_relax(m, l, 10); return; }
    int n = fas_n(m, l), nc = n / 2; long S = n + 4, Sc = nc + 4;
    double dx = fas_dx(m, l), dcx = fas_dx(m, l - 1), dc[6], dcc[6];
    fas_coefs(dx, dc);
    fas_coefs(dcx, dcc);
    fas_relax(m, l, 6);
    /* averageDown(crseState, state): AvgDown(2), children in Box([0,1]^3) order */
    double* uc = m->u[l-1];
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nc; z++) for (int y = 0; y < nc; y++) for (int x = 0; x < nc; x++) {
        double acc = 0.0;
        for (int kz = 0; kz < 2; kz++) for (int ky = 0; ky < 2; ky++) for (int kx = 0; kx < 2; kx++)
            acc = acc + 0.125 * m->u[l][IDX(2*x+kx+2, 2*y+ky+2, 2*z+kz+2, S)];
        uc[IDX(x+2, y+2, z+2, Sc)] = acc;
        m->c0[l-1][IDX(x, y, z, nc)] = acc;
    }
    /* coarseForce */
    fill_periodic(m->u[l], n, 2);
    fill_periodic(uc, nc, 2);
    fas_op(m->u[l], n, dx, dc, m->t[l]);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nc; z++) for (int y = 0; y < nc; y++) for (int x = 0; x < nc; x++) {
        double acc = 0.0;
        for (int kz = 0; kz < 2; kz++) for (int ky = 0; ky < 2; ky++) for (int kx = 0; kx < 2; kx++) {
            long o = IDX(2*x+kx, 2*y+ky, 2*z+kz, n);
            double res = m->t[l][o] + m->f[l][o];
            acc = acc + 0.125 * res;
        }
        m->f[l-1][IDX(x, y, z, nc)] = acc;
    }
    fas_op(uc, nc, dcx, dcc, m->t[l-1]);
    for (long o = 0; o < (long)nc*nc*nc; o++) m->f[l-1][o] = m->f[l-1][o] - m->t[l-1][o];
    fas_vcycle(m, l - 1);
    /* fineCorrect: c0 = -(c0 - crse); fine += 1.0 * c0(p/2) */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nc; z++) for (int y = 0; y < nc; y++) for (int x = 0; x < nc; x++) {
        long o = IDX(x, y, z, nc);
        m->c0[l-1][o] = (m->c0[l-1][o] - uc[IDX(x+2, y+2, z+2, Sc)]) * -1.0;
    }
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
        long i = IDX(x+2, y+2, z+2, S);
        m->u[l][i] = m->u[l][i] + 1.0 * m->c0[l-1][IDX(x/2, y/2, z/2, nc)];
    }
    fas_relax(m, l, 6);
}

static double fas_resnorm(or_fas* m, int l)
{
    int n = fas_n(m, l);
    double dx = fas_dx(m, l), dc[6];
    fas_coefs(dx, dc);
    fill_periodic(m->u[l], n, 2);
    fas_op(m->u[l], n, dx, dc, m->t[l]);
    double best = 0.0;
    for (long o = 0; o < (long)n*n*n; o++) best = upd_abs(best, m->t[l][o] + m->f[l][o]);
    return best;
}

/* force, phi: N^3 (x fastest); numLevels as LevelMultigridSolver's; hist: maxIter+1 entries.
 * Returns the number of V-cycles run. */
int or_mg_fas(int N, int numLevels, int maxIter, double tol, const double* force, double* phi, double* hist)
{
    or_fas m;
    m.N = N; m.levels = numLevels;
    m.u = (double**)calloc(numLevels, sizeof(double*));
    m.f = (double**)calloc(numLevels, sizeof(double*));
    m.c0 = (double**)calloc(numLevels, sizeof(double*));
    m.t = (double**)calloc(numLevels, sizeof(double*));
    m.r = (double**)calloc(numLevels, sizeof(double*));
    for (int l = 0; l < numLevels; l++) {
        long n = fas_n(&m, l);
        m.u[l] = (double*)calloc((size_t)(n+4)*(n+4)*(n+4), sizeof(double));
        m.f[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
        m.c0[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
        m.t[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
        m.r[l] = (double*)calloc((size_t)n*n*n, sizeof(double));
    }
    int top = numLevels - 1;
    long S = N + 4;
    for (int z = 0; z < N; z++) for (int y = 0; y < N; y++) for (int x = 0; x < N; x++) {
        m.u[top][IDX(x+2, y+2, z+2, S)] = phi[IDX(x, y, z, N)];
        m.f[top][IDX(x, y, z, N)] = force[IDX(x, y, z, N)];
    }
    double r0 = fas_resnorm(&m, top);
    hist[0] = r0;
    int it = 0;
    while (it < maxIter) {
        fas_vcycle(&m, top);
        double r = fas_resnorm(&m, top);
        hist[++it] = r;
        if (r < tol * r0) break;
    }
    for (int z = 0; z < N; z++) for (int y = 0; y < N; y++) for (int x = 0; x < N; x++)
        phi[IDX(x, y, z, N)] = m.u[top][IDX(x+2, y+2, z+2, S)];
    for (int l = 0; l < numLevels; l++) { free(m.u[l]); free(m.f[l]); free(m.c0[l]); free(m.t[l]); free(m.r[l]); }
    free(m.u); free(m.f); free(m.c0); free(m.t); free(m.r);
    return it;
}

/* ---------------------------------------------------------------------------------------------
 * Plain method, small: out = a*L(u, 1/h^2) + b*u on [0,n-1]^3 with u on [-1,n]^3.
 * ------------------------------------------------------------------------------------------- */
int or_plain_apply(int n, const double* u, double* out, double h, double a, double b)
{
    long S = n + 2;
    double c[7]; scaled(LAP7_C, 7, 1.0 / (h * h), c);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < n; z++) for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
        long i = IDX(x+1, y+1, z+1, S);
        double lu = lap7(u, i, S, c, 0.0);
        out[IDX(x, y, z, n)] = a * lu + b * u[i];
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Forward-Euler steps u += dt * L13(u, 1/h^2) on a periodic Lx*Ly*Lz domain held as one array
 * with ghost width 2 (a patch layout tiling that domain gives bitwise the same values, because
 * the ghost fill is exact and the update is pointwise). L13 = sum_d Derivative(2,d,4) in its
 * insertion order: +e, 0, -e, +2e, -2e per axis, the centre merged
 * (include/base/implem/Proto_StencilDefs.H:393-457). coefs/offs: the 13 terms as tabulated.
 * ------------------------------------------------------------------------------------------- */
int or_periodic_steps(int Lx, int Ly, int Lz, int g, const double* coefs, const int* offs, int n,
                      double h, double dt, int steps, double* u)
{
    long Sx = Lx + 2*g, Sy = Ly + 2*g, Sz = Lz + 2*g;
    double hsqinv = 1.0 / (h * h);
    double* c = (double*)malloc(sizeof(double) * n);
    long* lo = (long*)malloc(sizeof(long) * n);
    for (int j = 0; j < n; j++) { c[j] = (hsqinv != 1.0) ? coefs[j]*hsqinv : coefs[j]; lo[j] = offs[3*j] + Sx*(offs[3*j+1] + Sy*(long)offs[3*j+2]); }
    double* lu = (double*)malloc(sizeof(double) * (size_t)Lx*Ly*Lz);
    for (int s = 0; s < steps; s++) {
        #pragma omp parallel for collapse(2) schedule(static)
        for (long z = 0; z < Sz; z++) for (long y = 0; y < Sy; y++) for (long x = 0; x < Sx; x++) {
            if (x >= g && x < Lx+g && y >= g && y < Ly+g && z >= g && z < Lz+g) continue;
            long qx = ((x - g) % Lx + Lx) % Lx + g, qy = ((y - g) % Ly + Ly) % Ly + g, qz = ((z - g) % Lz + Lz) % Lz + g;
            u[x + Sx*(y + Sy*z)] = u[qx + Sx*(qy + Sy*qz)];
        }
        #pragma omp parallel for collapse(2) schedule(static)
        for (long z = 0; z < Lz; z++) for (long y = 0; y < Ly; y++) for (long x = 0; x < Lx; x++) {
            long i = (x+g) + Sx*((y+g) + Sy*(z+g));
            double acc = 0.0;
            for (int j = 0; j < n; j++) acc = acc + c[j] * u[i + lo[j]];
            lu[x + Lx*(y + Ly*z)] = acc;
        }
        #pragma omp parallel for collapse(2) schedule(static)
        for (long z = 0; z < Lz; z++) for (long y = 0; y < Ly; y++) for (long x = 0; x < Lx; x++) {
            long i = (x+g) + Sx*((y+g) + Sy*(z+g));
            u[i] += dt * lu[x + Lx*(y + Ly*z)];
        }
    }
    free(c); free(lo); free(lu);
    return 0;
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
