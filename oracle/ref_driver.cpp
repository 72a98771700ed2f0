// Reference-built oracle: the reference's own header-only C++ (Proto, DIM=3, HOST memory) compiled
// into a shared library, so that golden vectors and CPU baselines come from the reference code itself.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
// reference arm may load the library built from this file. Nothing on the product path uses it.
//
// Build: oracle/build_oracle.py (compiles this one translation unit against the reference's
// include/, include/base/, include/utils/, examples/_common/ and examples/_archived/LevelMultigrid/src
// where they lie, and writes oracle/_ref/libproto_ref.so). Every entry point is extern "C" with plain
// pointers so that Python's ctypes can call it.
//
// Reference code exercised (paths relative to the reference project root):
//   Stencil library + hostApply ........ include/base/implem/Proto_StencilDefs.H, Proto_StencilImplem.H:725-828
//   InterpStencil::Constant/Linear/Quadratic include/base/implem/Proto_InterpStencilDefs.H:1-80
//   LevelBoxData::exchange ............. include/base/implem/Proto_LevelBoxDataImplem.H:315-329, 900-951
//   Reduction<T,OP,HOST> ............... include/base/implem/Proto_ReductionImplem.H:62-101
//   LevelMultigrid (archived, 7-pt CS) . examples/_archived/LevelMultigrid/src/LevelMultigrid.cpp
//   LevelMultigridSolver (FAS, 13-pt) .. include/utils/implem/Proto_LevelMultigridSolverImplem.H
//                                        with examples/_common/BoxOp_Laplace.H
#include "Proto.H"
#include "BoxOp_Laplace.H"
#include "LevelMultigrid.cpp"   // the archived solver, compiled from where it lies (include path)
#include <vector>
#include <cstring>
#include <cmath>
#include <chrono>

using namespace Proto;

namespace {

Box mkbox(const int* lo, const int* hi) { return Box(Point(lo[0], lo[1], lo[2]), Point(hi[0], hi[1], hi[2])); }

Stencil<double> build_stencil(const double* coefs, const int* offs, int n,
                              const int* meta /* srcRatio[3], dstRatio[3], dstShift[3] */)
{
    Stencil<double> S;
    for (int j = 0; j < n; j++) {
        S += coefs[j] * Shift(Point(offs[3*j], offs[3*j+1], offs[3*j+2]));
    }
    S.srcRatio()  = Point(meta[0], meta[1], meta[2]);
    S.destRatio() = Point(meta[3], meta[4], meta[5]);
    S.destShift() = Point(meta[6], meta[7], meta[8]);
    return S;
}

int dump_stencil(const Stencil<double>& S, double* coefs, int* offs, int* meta, int cap)
{
    int n = (int)S.size();
    if (n > cap) return -n;
    for (int j = 0; j < n; j++) {
        coefs[j] = S.coefs()[j];
        for (int d = 0; d < 3; d++) offs[3*j+d] = S.offsets()[j][d];
    }
    for (int d = 0; d < 3; d++) {
        meta[d] = S.srcRatio()[d];
        meta[3+d] = S.destRatio()[d];
        meta[6+d] = S.destShift()[d];
    }
    return n;
}

// Copy a domain-sized array (x fastest over domainBox) into the valid cells of every patch.
template<typename LBD>
void load_level(LBD& lbd, const Box& domainBox, const double* in)
{
    for (auto dit : lbd.layout()) {
        auto& bd = lbd[dit];
        Box b = lbd.layout()[dit];
        for (auto it = b.begin(); it != b.end(); ++it) {
            bd(*it, 0) = in[domainBox.index(*it)];
        }
    }
}

template<typename LBD>
void store_level(const LBD& lbd, const Box& domainBox, double* out)
{
    for (auto dit : lbd.layout()) {
        const auto& bd = lbd[dit];
        Box b = lbd.layout()[dit];
        for (auto it = b.begin(); it != b.end(); ++it) {
            out[domainBox.index(*it)] = bd(*it, 0);
        }
    }
}

} // namespace

PROTO_KERNEL_START void f_axpbyT(Var<double> a_out, Var<double> a_lu, Var<double> a_u, double a_a, double a_b)
{
    a_out(0) = a_a*a_lu(0) + a_b*a_u(0);
}
PROTO_KERNEL_END(f_axpbyT, f_axpby)

PROTO_KERNEL_START void f_eulerT(Var<double> a_u, Var<double> a_lu, double a_dt)
{
    a_u(0) += a_dt*a_lu(0);
}
PROTO_KERNEL_END(f_eulerT, f_euler)

struct CSParams { int nu1, nu2, nuBottom; double omega; double beta; };

class RefCS {
public:
    RefCS(const DisjointBoxLayout& layout, double dx, int level, const CSParams& p, bool helm)
        : m_layout(layout), m_dx(dx), m_level(level), m_p(p), m_helm(helm)
    {
        m_alpha.define(layout, Point::Zeros());
        m_alpha.setToZero();
        if (level > 0) {
            Point r = Point::Ones(2);
            DisjointBoxLayout crseLocal = layout.coarsen(r);
            ProblemDomain pdc = layout.domain().coarsen(r);
            DisjointBoxLayout crse;
            Point bs = layout.boxSize();
            if (pdc.sizes() % bs == Point::Zeros()) crse = DisjointBoxLayout(pdc, bs);
            else crse = DisjointBoxLayout(pdc, pdc.sizes());
            m_resc.define(crse, Point::Zeros());
            m_delta.define(crse, Point::Ones());
            m_local.define(crseLocal, Point::Zeros());
            m_crse = std::make_shared<RefCS>(crse, 2*dx, level-1, p, helm);
        }
    }
    LevelBoxData<double>& alpha() { return m_alpha; }
    void restrictAlpha() {
        if (m_level == 0 || !m_helm) return;
        auto A = Stencil<double>::AvgDown(2);
        for (auto dit : m_alpha) { m_local[dit] |= A(m_alpha[dit]); }
        m_local.copyTo(m_crse->m_alpha);
        m_crse->restrictAlpha();
    }
    // res = f - A phi (Helmholtz) or rho + L(phi, -1/h^2) (Poisson), on the valid box
    void residual(BoxData<double>& res, BoxData<double>& phi, BoxData<double>& rhs, BoxData<double>& alpha) {
        auto L = Stencil<double>::Laplacian();
        double hsqinv = 1./(m_dx*m_dx);
        if (!m_helm) {
            res.setVal(0.);
            res += rhs;
            res += L(phi, -hsqinv);
        } else {
            BoxData<double> lphi(res.box());
            lphi |= L(phi, hsqinv);
            double beta = m_p.beta;
            forallInPlace([] PROTO_LAMBDA (Var<double> r, Var<double> lp, Var<double> ph, Var<double> f,
                                           Var<double> al, double be) {
                r(0) = f(0) - (al(0)*ph(0) - be*lp(0));
            }, res, lphi, phi, rhs, alpha, beta);
        }
    }
    double resnorm(LevelBoxData<double>& phi, LevelBoxData<double>& rhs) {
        phi.exchange();
        Reduction<double, Abs> rxn;
        double hsqinv = 1./(m_dx*m_dx);
        auto L = Stencil<double>::Laplacian();
        for (auto dit : phi) {
            BoxData<double> res(phi.layout()[dit]);
            if (!m_helm) {
                res.setVal(0.);
                res -= rhs[dit];
                res += L(phi[dit], hsqinv);
            } else {
                residual(res, phi[dit], rhs[dit], m_alpha[dit]);
            }
            res.reduce(rxn);
        }
        return rxn.fetch();
    }
    void relax(LevelBoxData<double>& phi, LevelBoxData<double>& rhs, int n) {
        auto L = Stencil<double>::Laplacian();
        double w = m_p.omega/6.0;
        double lambda = (m_p.omega*(m_dx*m_dx))/6.0;
        Stencil<double> D = (-lambda)*Shift(Point::Zeros());
        double hsqinv = 1./(m_dx*m_dx);
        double diagB = 6.0*m_p.beta*hsqinv;
        for (int k = 0; k < n; k++) {
            phi.exchange();
            for (auto dit : phi) {
                BoxData<double>& p = phi[dit];
                BoxData<double>& r = rhs[dit];
                if (!m_helm) {
                    BoxData<double> temp = L(p, w);
                    temp += D(r);
                    p += temp;
                } else {
                    BoxData<double> res(phi.layout()[dit]);
                    residual(res, p, r, m_alpha[dit]);
                    double om = m_p.omega;
                    forallInPlace([] PROTO_LAMBDA (Var<double> ph, Var<double> rs, Var<double> al,
                                                   double omg, double db) {
                        ph(0) = ph(0) + (omg*rs(0))/(al(0) + db);
                    }, p, res, m_alpha[dit], om, diagB);
                }
            }
        }
    }
    void coarseResidual(LevelBoxData<double>& resc, LevelBoxData<double>& phi, LevelBoxData<double>& rhs) {
        phi.exchange();
        auto A = Stencil<double>::AvgDown(2);
        for (auto dit : phi) {
            BoxData<double> res(phi.layout()[dit]);
            residual(res, phi[dit], rhs[dit], m_alpha[dit]);
            m_local[dit] |= A(res);
        }
        m_local.copyTo(resc);
    }
    void fineInterp(LevelBoxData<double>& phi, LevelBoxData<double>& delta) {
        delta.copyTo(m_local);
        auto I = InterpStencil<double>::Constant(Point::Ones(2));
        for (auto dit : phi) { phi[dit] += I(m_local[dit]); }
    }
    void vCycle(LevelBoxData<double>& phi, LevelBoxData<double>& rhs) {
        if (m_level > 0) {
            relax(phi, rhs, m_p.nu1);
            coarseResidual(m_resc, phi, rhs);
            m_delta.setToZero();
            m_crse->vCycle(m_delta, m_resc);
            fineInterp(phi, m_delta);
            relax(phi, rhs, m_p.nu2);
        } else {
            relax(phi, rhs, m_p.nuBottom);
        }
    }
private:
    DisjointBoxLayout m_layout;
    double m_dx;
    int m_level;
    CSParams m_p;
    bool m_helm;
    LevelBoxData<double> m_resc, m_delta, m_local, m_alpha;
    std::shared_ptr<RefCS> m_crse;
};

extern "C" {

// ---- stencil library tables -----------------------------------------------------------------
// which: 0 Laplacian, 1 Laplacian_19, 2 Laplacian_27, 3 Derivative(a,b,c), 4 AvgDown(a),
//        5 DiffCellToFace(a, side=b, order=c), 6 sum_d Derivative(2,d,4) (13-point Laplacian),
//        7 CellToFace(a, side=b, order=c), 8 FluxDivergence(a), 9 Sum(a), 10 LaplacianFace(a, b),
//        11 faceToCell(a, b), 12 Identity (1.0*Shift::Zeros()), 13 CornersToCells(a)
int ref_stencil_table(int which, int a, int b, int c, double* coefs, int* offs, int* meta, int cap)
{
    Stencil<double> S;
    switch (which) {
        case 0: S = Stencil<double>::Laplacian(); break;
        case 1: S = Stencil<double>::Laplacian_19(); break;
        case 2: S = Stencil<double>::Laplacian_27(); break;
        case 3: S = Stencil<double>::Derivative(a, b, c); break;
        case 4: S = Stencil<double>::AvgDown(a); break;
        case 5: S = Stencil<double>::DiffCellToFace(a, b ? Side::Hi : Side::Lo, c); break;
        case 6: {
            S = Stencil<double>::Derivative(2, 0, 4);
            for (int d = 1; d < DIM; d++) S += Stencil<double>::Derivative(2, d, 4);
            break;
        }
        case 7: S = Stencil<double>::CellToFace(a, b ? Side::Hi : Side::Lo, c); break;
        case 8: S = Stencil<double>::FluxDivergence(a); break;
        case 9: S = Stencil<double>::Sum(a); break;
        case 10: S = Stencil<double>::LaplacianFace(a, b); break;
        case 11: S = Stencil<double>::faceToCell(a, b); break;
        case 12: S = 1.0*Shift::Zeros(); break;
        case 13: S = Stencil<double>::CornersToCells(a); break;
        default: return 0;
    }
    return dump_stencil(S, coefs, offs, meta, cap);
}

// ---- Stencil apply through the public operators ---------------------------------------------
// mode: 0 "dst |= S(src, scale)", 1 "dst += S(src, scale)",
//       2 "dst |= S(src, range, scale)", 3 "dst += S(src, range, scale)".
int ref_stencil_apply(const double* coefs, const int* offs, int n, const int* meta,
                      const double* src, const int* srcLo, const int* srcHi,
                      double* dst, const int* dstLo, const int* dstHi,
                      const int* rLo, const int* rHi, int mode, double scale, int ncomp)
{
    Stencil<double> S = build_stencil(coefs, offs, n, meta);
    Box sb = mkbox(srcLo, srcHi), db = mkbox(dstLo, dstHi);
    if (ncomp == 1) {
        BoxData<double,1,HOST> s(src, sb, 1), d(dst, db, 1);
        switch (mode) {
            case 0: d |= S(s, scale); break;
            case 1: d += S(s, scale); break;
            case 2: d |= S(s, mkbox(rLo, rHi), scale); break;
            case 3: d += S(s, mkbox(rLo, rHi), scale); break;
            default: return -1;
        }
    } else if (ncomp == 3) {
        BoxData<double,3,HOST> s(src, sb, 3), d(dst, db, 3);
        switch (mode) {
            case 0: d |= S(s, scale); break;
            case 1: d += S(s, scale); break;
            case 2: d |= S(s, mkbox(rLo, rHi), scale); break;
            case 3: d += S(s, mkbox(rLo, rHi), scale); break;
            default: return -1;
        }
    } else {
        return -2;
    }
    return 0;
}

// Output box the reference infers for "BoxData out = S(src)" (LazyStencil::inferredRange).
int ref_stencil_range(const double* coefs, const int* offs, int n, const int* meta,
                      const int* srcLo, const int* srcHi, int* outLo, int* outHi)
{
    Stencil<double> S = build_stencil(coefs, offs, n, meta);
    Box r = S.range(mkbox(srcLo, srcHi));
    for (int d = 0; d < 3; d++) { outLo[d] = r.low()[d]; outHi[d] = r.high()[d]; }
    return r.empty() ? 1 : 0;
}

// Box algebra probes (bit-exact index work): op 0 coarsen(ratio), 1 taperCoarsen(ratio), 2 refine(ratio)
int ref_box_op(int op, const int* lo, const int* hi, const int* ratio, int* outLo, int* outHi)
{
    Box b = mkbox(lo, hi);
    Point r(ratio[0], ratio[1], ratio[2]);
    Box o;
    switch (op) {
        case 0: o = b.coarsen(r); break;
        case 1: o = b.taperCoarsen(r); break;
        case 2: o = b.refine(r); break;
        default: return -1;
    }
    for (int d = 0; d < 3; d++) { outLo[d] = o.low()[d]; outHi[d] = o.high()[d]; }
    return 0;
}

// ---- InterpStencil: kind 0 Constant, 1 Linear; "dst |= I(src, scale)" or "dst += I(src, scale)"
int ref_interp_apply(int kind, int ratio, const double* src, const int* srcLo, const int* srcHi,
                     double* dst, const int* dstLo, const int* dstHi, int overwrite, double scale)
{
    InterpStencil<double> I = (kind == 0) ? InterpStencil<double>::Constant(Point::Ones(ratio))
                            : (kind == 1) ? InterpStencil<double>::Linear(Point::Ones(ratio))
                                          : InterpStencil<double>::Quadratic(Point::Ones(ratio));
    BoxData<double,1,HOST> s(src, mkbox(srcLo, srcHi), 1), d(dst, mkbox(dstLo, dstHi), 1);
    if (overwrite) d |= I(s, scale); else d += I(s, scale);
    return 0;
}

// ---- LevelBoxData exchange on a uniform layout --------------------------------------------------
// valid: domain array (x fastest). out: for every patch in lexicographic patch order (x fastest),
// the patch's grown BoxData (box grown by ghost), x fastest. Ghost cells start at 'fill'.
int ref_exchange(const int* domainSize, const int* periodic, const int* boxSize, const int* ghost,
                 const double* valid, double* out, double fill)
{
    Box domainBox(Point::Zeros(), Point(domainSize[0]-1, domainSize[1]-1, domainSize[2]-1));
    Array<bool, DIM> per;
    for (int d = 0; d < 3; d++) per[d] = periodic[d] != 0;
    ProblemDomain pd(domainBox, per);
    DisjointBoxLayout layout(pd, Point(boxSize[0], boxSize[1], boxSize[2]));
    Point g(ghost[0], ghost[1], ghost[2]);
    LevelBoxData<double,1,HOST> lbd(layout, g);
    for (auto dit : layout) lbd[dit].setVal(fill);
    load_level(lbd, domainBox, valid);
    lbd.exchange();
    int np[3];
    for (int d = 0; d < 3; d++) np[d] = domainSize[d] / boxSize[d];
    size_t patchVol = (size_t)(boxSize[0]+2*ghost[0])*(boxSize[1]+2*ghost[1])*(boxSize[2]+2*ghost[2]);
    for (auto dit : layout) {
        Box b = layout[dit];
        int px = b.low()[0]/boxSize[0], py = b.low()[1]/boxSize[1], pz = b.low()[2]/boxSize[2];
        size_t pidx = (size_t)px + (size_t)np[0]*((size_t)py + (size_t)np[1]*pz);
        const auto& bd = lbd[dit];
        Box gb = bd.box();
        double* o = out + pidx*patchVol;
        for (auto it = gb.begin(); it != gb.end(); ++it) o[gb.index(*it)] = bd(*it, 0);
    }
    return 0;
}

// ---- reductions: op 0 Max, 1 Min, 2 Abs (absMax), 3 Sum, 4 SumAbs, 5 SumSquare ------------------
double ref_reduce(int op, const double* data, int n)
{
    BoxData<double,1,HOST> b(data, Box(Point::Zeros(), Point(n-1, 0, 0)), 1);
    switch (op) {
        case 0: { Reduction<double, Max, HOST> r; b.reduce(r); return r.fetch(); }
        case 1: { Reduction<double, Min, HOST> r; b.reduce(r); return r.fetch(); }
        case 2: { Reduction<double, Abs, HOST> r; b.reduce(r); return r.fetch(); }
        case 3: { Reduction<double, Sum, HOST> r; b.reduce(r); return r.fetch(); }
        case 4: { Reduction<double, SumAbs, HOST> r; b.reduce(r); return r.fetch(); }
        case 5: { Reduction<double, SumSquare, HOST> r; b.reduce(r); return r.fetch(); }
    }
    return 0.0;
}

// ---- plain method, small: out = a*L(u) + b*u on [0,n-1]^3, u on [-1,n]^3 ---------------------

int ref_plain_apply(int n, const double* u, double* out, double h, double a, double b)
{
    Box inner = Box::Cube(n);
    BoxData<double,1,HOST> U(u, inner.grow(1), 1);
    BoxData<double,1,HOST> O(out, inner, 1);
    auto L = Stencil<double>::Laplacian();
    BoxData<double,1,HOST> LU = L(U, 1.0/(h*h));
    forallInPlace(f_axpby, O, LU, U, a, b);
    return 0;
}

// ---- archived 7-point correction-scheme multigrid, unmodified -------------------------------
// rho/phi: domain arrays (x fastest, N^3). numLevels as the archived driver's "numLevels"
// argument (the solver holds levels numLevels..0). Returns the number of V-cycles run.
int ref_mg_archived(int N, int boxSize, int numLevels, int maxIter, double tol,
                    const double* rho, double* phi, double* hist)
{
    Box domain = Box::Cube(N);
    Array<bool,DIM> per; per.fill(true);
    double dx = 1.0/N;
    ProblemDomain pd(domain, per);
    DisjointBoxLayout layout(pd, Point::Ones(boxSize));
    LevelBoxData<double> R(layout, Point::Zeros());
    LevelBoxData<double> P(layout, Point::Ones());
    R.setToZero(); P.setToZero();
    load_level(R, domain, rho);
    load_level(P, domain, phi);
    LevelMultigrid mg(layout, dx, numLevels);
    double r0 = mg.resnorm(P, R);
    hist[0] = r0;
    int it = 0;
    for (; it < maxIter; ) {
        mg.vCycle(P, R);
        double r = mg.resnorm(P, R);
        hist[++it] = r;
        if (r < tol*r0) break;
    }
    store_level(P, domain, phi);
    return it;
}

// ---- LevelMultigridSolver<BoxOp_Laplace> (FAS, 4th-order flux-form operator), unmodified ------
// The solver's own solve() is driven one V-cycle at a time to record the residual history; each
// call recomputes the initial residual (no state change) before its single V-cycle.
int ref_mg_fas(int N, int boxSize, int numLevels, int maxIter, double tol,
               const double* force, double* phi, double* hist)
{
    Box domain = Box::Cube(N);
    Array<bool,DIM> per; per.fill(true);
    double dx = 1.0/N;
    ProblemDomain pd(domain, per);
    DisjointBoxLayout layout(pd, Point::Ones(boxSize));
    typedef BoxOp_Laplace<double> OP;
    LevelMultigridSolver<BoxOp_Laplace, double> solver(layout, Point::Ones(2), numLevels, dx);
    LevelBoxData<double, 1> Phi(layout, OP::ghost());
    LevelBoxData<double, 1> G(layout, Point::Zeros());
    Phi.setToZero(); G.setToZero();
    load_level(G, domain, force);
    load_level(Phi, domain, phi);
    LevelBoxData<double, 1> Res(layout, Point::Zeros());
    double r0 = solver.resnorm(Res, Phi, G);
    hist[0] = r0;
    int it = 0;
    for (; it < maxIter; ) {
        double r = solver.solve(Phi, G, 1, tol);
        hist[++it] = r;
        if (r < tol*r0) break;
    }
    store_level(Phi, domain, phi);
    return it;
}

// ---- parameterised correction-scheme multigrid on reference primitives -----------------------
// Same structure as the archived solver (relax / coarse residual / average / constant prolong),
// with the smoother weight and sweep counts as parameters and an optional per-cell Helmholtz
// coefficient. Equation: alpha*u - beta*L_h u = f.
//   Poisson form (alpha == nullptr): written in the archived sign convention, L_h phi = rho with
//   rho = -f/beta... here callers pass rho directly (beta ignored) and
//     relax:     phi += [ L(phi, w) + (-lambda)*rho ],  w = omega/6, lambda = omega*h*h/6
//     residual:  res = rho + L(phi, -1/h^2)        (coarse right-hand side: AvgDown(res))
//     resnorm:   max | -rho + L(phi, 1/h^2) |
//   Helmholtz form (alpha != nullptr, beta > 0), per cell:
//     Lphi = L(phi, 1/h^2);  r = f - (alpha*phi - beta*Lphi);  phi += (omega*r)/(alpha + 6*beta/h^2)
//     residual / resnorm use r; alpha on coarse levels is AvgDown(alpha).

// levels: index of the finest level (the solver holds levels..0, i.e. levels+1 grids).
// alpha == nullptr selects the Poisson form (rhs is rho in L_h phi = rho).
int ref_mg_cs(int N, int boxSize, int levels, int nu1, int nu2, int nuBottom, double omega,
              double beta, const double* alpha, int maxIter, double tol,
              const double* rhs, double* phi, double* hist)
{
    Box domain = Box::Cube(N);
    Array<bool,DIM> per; per.fill(true);
    double dx = 1.0/N;
    ProblemDomain pd(domain, per);
    DisjointBoxLayout layout(pd, Point::Ones(boxSize));
    CSParams p{nu1, nu2, nuBottom, omega, beta};
    RefCS mg(layout, dx, levels, p, alpha != nullptr);
    LevelBoxData<double> R(layout, Point::Zeros());
    LevelBoxData<double> P(layout, Point::Ones());
    R.setToZero(); P.setToZero();
    load_level(R, domain, rhs);
    load_level(P, domain, phi);
    if (alpha) { load_level(mg.alpha(), domain, alpha); mg.restrictAlpha(); }
    double r0 = mg.resnorm(P, R);
    hist[0] = r0;
    int it = 0;
    for (; it < maxIter; ) {
        mg.vCycle(P, R);
        double r = mg.resnorm(P, R);
        hist[++it] = r;
        if (r < tol*r0) break;
    }
    store_level(P, domain, phi);
    return it;
}

// Time 'reps' V-cycles (+ residual norms) of ref_mg_cs's solver on an N^3 grid; returns seconds.
double ref_mg_cs_time_cycles(int N, int boxSize, int levels, int nu1, int nu2, int nuBottom,
                             double omega, const double* rhs, int reps)
{
    Box domain = Box::Cube(N);
    Array<bool,DIM> per; per.fill(true);
    double dx = 1.0/N;
    ProblemDomain pd(domain, per);
    DisjointBoxLayout layout(pd, Point::Ones(boxSize));
    CSParams p{nu1, nu2, nuBottom, omega, 1.0};
    RefCS mg(layout, dx, levels, p, false);
    LevelBoxData<double> R(layout, Point::Zeros());
    LevelBoxData<double> P(layout, Point::Ones());
    R.setToZero(); P.setToZero();
    load_level(R, domain, rhs);
    auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < reps; k++) { mg.vCycle(P, R); (void)mg.resnorm(P, R); }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Runs ncycles V-cycles of ref_mg_cs's Poisson solver from phi = 0, each followed by the residual
// norm, exactly as a solve does; when a solve reaches res < tol*res0 the next cycle starts a new
// solve from phi = 0 (its initial norm counted in that cycle). *t_start is the steady-clock time
// (seconds) before the first norm, t_end[k] the time at which cycle k ended. Returns the number of
// cycles the first solve took to converge (0 if none converged within ncycles).
int ref_mg_cs_cycles(int N, int boxSize, int levels, int nu1, int nu2, int nuBottom, double omega,
                     double tol, const double* rhs, int ncycles, double* t_start, double* t_end,
                     int* solves_done)
{
    auto now = []() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    };
    Box domain = Box::Cube(N);
    Array<bool,DIM> per; per.fill(true);
    double dx = 1.0/N;
    ProblemDomain pd(domain, per);
    DisjointBoxLayout layout(pd, Point::Ones(boxSize));
    CSParams p{nu1, nu2, nuBottom, omega, 1.0};
    RefCS mg(layout, dx, levels, p, false);
    LevelBoxData<double> R(layout, Point::Zeros());
    LevelBoxData<double> P(layout, Point::Ones());
    R.setToZero(); P.setToZero();
    load_level(R, domain, rhs);
    *t_start = now();
    double r0 = mg.resnorm(P, R);
    int first = 0, done = 0, inSolve = 0;
    for (int k = 0; k < ncycles; k++) {
        if (inSolve < 0) {          // previous solve converged: start the next one from zero
            P.setToZero();
            r0 = mg.resnorm(P, R);
            inSolve = 0;
        }
        mg.vCycle(P, R);
        double r = mg.resnorm(P, R);
        inSolve++;
        if (r < tol*r0) {
            if (done == 0) first = inSolve;
            done++;
            inSolve = -1;
        }
        t_end[k] = now();
    }
    *solves_done = done;
    return first;
}

// BoxOp_Laplace::operator()(output, state, scale) of the reference on one box (state and output alias
// caller memory), with the flux scale set through BoxOp::setFluxScale.
int ref_boxop_laplace(const double* u, const int* sLo, const int* sHi, double* out, const int* oLo, const int* oHi,
                      double dx, double fluxScale, double scale)
{
    Box sb = mkbox(sLo, sHi), ob = mkbox(oLo, oHi);
    BoxData<double,1,HOST> state(const_cast<double*>(u), sb, 1);
    BoxData<double,1,HOST> output(out, ob, 1);
    // the operator is defined on a one-box layout of the output box (it only keeps dx from it)
    Array<bool,DIM> per; per.fill(false);
    ProblemDomain pd(ob, per);
    DisjointBoxLayout layout(pd, ob.sizes());
    BoxOp_Laplace<double,HOST> op;
    op.define(layout, *layout.begin(), dx);
    op.setFluxScale(fluxScale);
    op(output, state, scale);
    return 0;
}

// ---- AMR-level stepping on uneven patches (per-patch BoxData, ghost fill by BoxData::copyTo) ----
// Patches tile a periodic domain as a tensor product of per-axis widths. For every step:
// periodic ghost fill, Lu = L13(u, 1/h^2) (13-point: sum_d Derivative(2,d,4)), u += dt*Lu.
// data: concatenation of every patch's grown BoxData (x fastest; patch order x fastest).

int ref_level13_steps(const int* nx, const int* ny, const int* nz, const int* counts, int ghost,
                      double h, double dt, int steps, double* data)
{
    std::vector<int> w[3];
    const int* widths[3] = {nx, ny, nz};
    int L[3];
    for (int d = 0; d < 3; d++) {
        L[d] = 0;
        for (int k = 0; k < counts[d]; k++) { w[d].push_back(widths[d][k]); L[d] += widths[d][k]; }
    }
    std::vector<Box> boxes;
    std::vector<std::shared_ptr<BoxData<double,1,HOST>>> bds;
    size_t off = 0;
    int z0 = 0;
    for (int k = 0; k < counts[2]; k++) {
        int y0 = 0;
        for (int j = 0; j < counts[1]; j++) {
            int x0 = 0;
            for (int i = 0; i < counts[0]; i++) {
                Box b(Point(x0, y0, z0), Point(x0 + w[0][i] - 1, y0 + w[1][j] - 1, z0 + w[2][k] - 1));
                boxes.push_back(b);
                Box gb = b.grow(ghost);
                bds.push_back(std::make_shared<BoxData<double,1,HOST>>(data + off, gb, 1));
                off += gb.size();
                x0 += w[0][i];
            }
            y0 += w[1][j];
        }
        z0 += w[2][k];
    }
    auto L13 = Stencil<double>::Derivative(2, 0, 4);
    for (int d = 1; d < DIM; d++) L13 += Stencil<double>::Derivative(2, d, 4);
    double hsqinv = 1.0/(h*h);
    size_t np = boxes.size();
    for (int s = 0; s < steps; s++) {
        // ghost fill: every patch's grown box takes the periodic images of all patches' valid cells
        for (size_t i = 0; i < np; i++) {
            Box gb = boxes[i].grow(ghost);
            for (size_t j = 0; j < np; j++) {
                for (int sz = -1; sz <= 1; sz++)
                for (int sy = -1; sy <= 1; sy++)
                for (int sx = -1; sx <= 1; sx++) {
                    if (i == j && sx == 0 && sy == 0 && sz == 0) continue;
                    Point sh(sx*L[0], sy*L[1], sz*L[2]);
                    Box img = boxes[j].shift(sh) & gb;
                    if (img.empty()) continue;
                    bds[j]->copyTo(*bds[i], img.shift(-sh), sh);
                }
            }
        }
        for (size_t i = 0; i < np; i++) {
            BoxData<double,1,HOST> lu(boxes[i]);
            lu |= L13(*bds[i], hsqinv);
            forallInPlace(f_euler, *bds[i], lu, dt);
        }
    }
    return 0;
}

// BoxPartition(patchDomain, patches, 0, nranks): Morton::sort, then loadBalance's contiguous
// segments (include/base/implem/Proto_BoxPartitionImplem.H:35-54,196-222). owner[i] is the process
// of points[i] (input order). The patch domain is the bounding box of the points, periodic.
int ref_load_balance(const int* points, int n, int nranks, int* owner)
{
    if (n <= 0 || nranks <= 0) return -1;
    std::vector<Point> pts;
    Point hi = Point::Zeros();
    for (int i = 0; i < n; i++) {
        Point p(points[3*i], points[3*i+1], points[3*i+2]);
        pts.push_back(p);
        for (int d = 0; d < 3; d++) if (p[d] > hi[d]) hi[d] = p[d];
    }
    ProblemDomain pd(Box(Point::Zeros(), hi), true);
    BoxPartition part(pd, pts, 0, (unsigned int)nranks);
    const auto& assigned = part.partition();
    if ((int)assigned.size() != n) return -2;
    for (int i = 0; i < n; i++) {
        owner[i] = -1;
        for (const auto& a : assigned) if (a.first == pts[i]) { owner[i] = (int)a.second; break; }
        if (owner[i] < 0) return -3;
    }
    return 0;
}

} // extern "C"
