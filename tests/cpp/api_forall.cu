// The forall family, BoxOp_Laplace, LevelOp (with the library's operator and with a user operator
// plugged in) and the reference-signature multigrid solvers, written like the reference's own tests
// (tests/ForallTests.cpp, tests/LevelOpTests.cpp, the archived LevelMultigrid driver). Compiled
// with nvcc; writes every result to argv[2] for the checks in tests/test_cpp_api.py.
#include <cmath>
#include <cstdio>
#include <vector>

#include "proto_b200/cpp/Proto_B200_Forall.cuh"

using namespace Proto;
#define DIM 3

PROTO_KERNEL_START
void consToPrim_temp(Var<double, DIM + 2>& W, const Var<double, DIM + 2>& U, double gamma)
{
    double rho = U(0);
    double v, v2 = 0.;
    W(0) = rho;
    for (int i = 1; i <= DIM; i++) {
        v = U(i) / rho;
        W(i) = v;
        v2 += v * v;
    }
    W(DIM + 1) = (U(DIM + 1) - .5 * rho * v2) * (gamma - 1.);
}
PROTO_KERNEL_END(consToPrim_temp, consToPrim)

PROTO_KERNEL_START
void sineFunc_temp(Point& a_p, Var<double>& a_Y, const Var<double, DIM>& a_X, double phase)
{
    a_Y(0) = 0.0;
    for (int ii = 0; ii < DIM; ii++) a_Y(0) += sin(a_X(ii) + phase);
    a_Y(0) += 0.001 * (a_p[0] + 10 * a_p[1] + 100 * a_p[2]);
}
PROTO_KERNEL_END(sineFunc_temp, sineFunc)

PROTO_KERNEL_START
void iota_temp(Point& a_p, Var<double, DIM + 2>& a_U)
{
    for (int c = 0; c < DIM + 2; c++) a_U(c) = 1.0 + 0.25 * c + 0.01 * (a_p[0] + 2 * a_p[1] + 3 * a_p[2]);
}
PROTO_KERNEL_END(iota_temp, iota)

// a user operator for LevelOp: the 7-point Laplacian through the Stencil API
template <typename T, MemType MEM>
struct MyLaplace7 {
    double m_dx = 1.0;
    void define(double dx) { m_dx = dx; }
    double spectralRadius() const { return 12.0 / (m_dx * m_dx); }
    void operator()(BoxData<T, 1, MEM>& out, const BoxData<T, 1, MEM>& state, T scale = 1.0) const
    {
        out |= Stencil<T>::Laplacian()(state, scale / (m_dx * m_dx));
    }
};

static std::vector<double> g_out;
template <unsigned int C>
static void emit(const BoxData<double, C>& b)
{
    std::vector<double> h;
    b.copyToHost(h);
    g_out.insert(g_out.end(), h.begin(), h.end());
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const double gamma = 1.4, phase = M_PI / 4.;
    // 1. forall: consToPrim on U (iota-filled by forall_p), on U's box and on a given box
    Box srcBox = Box::Cube(4);
    BoxData<double, DIM + 2> U = forall_p<double, DIM + 2>(iota, srcBox);
    emit(U);
    BoxData<double, DIM + 2> W = forall<double, DIM + 2>(consToPrim, U, gamma);
    if (W.box() != U.box()) return 10;
    emit(W);
    Box destBox = Box::Cube(3);
    BoxData<double, DIM + 2> W2 = forall<double, DIM + 2>(consToPrim, destBox, U, gamma);
    if (W2.box() != destBox) return 11;
    emit(W2);
    // 2. forallInPlace on the intersection, then on a compute box
    BoxData<double, DIM + 2> W3(destBox, 0.0);
    forallInPlace(consToPrim, W3, U, gamma);
    emit(W3);
    BoxData<double, DIM + 2> W4(destBox, -7.0);
    forallInPlace(consToPrim, Box::Cube(2), W4, U, gamma);
    emit(W4);
    // 3. forall_p / forallInPlace_p with a point-dependent function
    BoxData<double, DIM> X(srcBox, 1.0);
    forallInPlace_p([=] PROTO_LAMBDA (Point& p, Var<double, DIM>& x) {
        for (int d = 0; d < DIM; d++) x(d) = 0.1 * p[d] + 0.05 * d;
    }, X);
    emit(X);
    BoxData<double> Y = forall_p<double>(sineFunc, X, phase);
    emit(Y);
    BoxData<double> Y2 = forall_p<double>(sineFunc, destBox, X, phase);
    emit(Y2);
    BoxData<double> Y3(destBox, 3.0);
    forallInPlace_p(sineFunc, Box::Cube(2), Y3, X, phase);
    emit(Y3);
    // 4. a lambda update u += dt * lu (the AMR-level step's pointwise part), forallOp form
    BoxData<double> u = forall_p<double>([=] PROTO_LAMBDA (Point& p, Var<double>& v) { v(0) = 0.5 * p[0] - 0.25 * p[2]; },
                                         srcBox);
    BoxData<double> lu(srcBox, 2.0);
    forallInPlaceOp(1, "euler", [=] PROTO_LAMBDA (Var<double>& a, const Var<double>& b, double dt) { a(0) += dt * b(0); },
                    u, lu, 0.125);
    emit(u);
    // 5. BoxOp_Laplace on a box with its ghost cells (flux scale -1, and a scale)
    const int n = 12;
    const double dx = 1.0 / n;
    Box valid = Box::Cube(n);
    BoxData<double> phi = forall_p<double>([=] PROTO_LAMBDA (Point& p, Var<double>& v) {
        v(0) = sin(0.3 * p[0] + 0.2 * p[1] * p[1] - 0.1 * p[2]);
    }, valid.grow(2));
    emit(phi);
    BoxOp_Laplace<double> op(dx);
    op.setFluxScale(-1.0);
    BoxData<double> lphi(valid);
    op(lphi, phi, 0.5);
    emit(lphi);
    // 6. LevelOp over a periodic 2x2x2 layout of 6^3 patches, ghost 2: the library's operator and a
    //    user operator plugged into the same LevelOp
    ProblemDomain pd(valid, true);
    DisjointBoxLayout layout(pd, Point::Ones(6));
    LevelBoxData<double> state(layout, Point::Ones(2)), lout(layout, Point::Ones(2)), lout7(layout, Point::Ones(2));
    for (size_t i = 0; i < state.size(); i++) {
        BoxData<double> s = state[i];
        phi.copyTo(s, layout[i]);
    }
    LevelOp<BoxOp_Laplace, double> lop(layout, dx);
    lop(lout, state);
    for (size_t i = 0; i < lout.size(); i++) emit(lout[i]);
    LevelOp<MyLaplace7, double> lop7(layout, dx);
    lop7(lout7, state);
    for (size_t i = 0; i < lout7.size(); i++) emit(lout7[i]);
    // 7. the archived LevelMultigrid with the reference's signature and driver loop
    const int N = 32;
    ProblemDomain pd2(Box::Cube(N), true);
    DisjointBoxLayout layout2(pd2, Point::Ones(16));
    LevelBoxData<double> rho(layout2, Point::Zeros()), psi(layout2, Point::Ones());
    rho.setToZero();
    psi.setToZero();
    for (size_t i = 0; i < rho.size(); i++) {
        BoxData<double> r = rho[i];
        forallInPlace_p([=] PROTO_LAMBDA (Point& p, Var<double>& v) {
            v(0) = cos(2 * M_PI * (p[0] + 0.5) / N) * sin(4 * M_PI * (p[1] + 0.5) / N) + 0.5 * sin(2 * M_PI * (p[2] + 0.5) / N);
        }, r);
    }
    LevelMultigrid mg(layout2, 1.0 / N, 3);
    double res0 = mg.resnorm(psi, rho);
    std::printf("mg res %d %.17g\n", 0, res0);
    for (int it = 0; it < 6; it++) {
        mg.vCycle(psi, rho);
        double r = mg.resnorm(psi, rho);
        std::printf("mg res %d %.17g\n", it + 1, r);
        if (r < 1e-10 * res0) break;
    }
    for (size_t i = 0; i < rho.size(); i++) emit(rho[i]);
    for (size_t i = 0; i < psi.size(); i++) emit(psi[i]);
    // 8. LevelMultigridSolver<BoxOp_Laplace, double> with the reference's signature
    LevelBoxData<double> st(layout2, Point::Ones(2)), force(layout2, Point::Zeros());
    st.setToZero();
    for (size_t i = 0; i < force.size(); i++) {
        BoxData<double> f = force[i];
        BoxData<double> r = rho[i];
        r.copyTo(f);
    }
    LevelMultigridSolver<BoxOp_Laplace, double> fas(layout2, Point::Ones(2), 4, 1.0 / N);
    double fr = fas.solve(st, force, 8, 1e-10);
    for (size_t k = 0; k < fas.history().size(); k++) std::printf("fas res %zu %.17g\n", k, fas.history()[k]);
    std::printf("fas final %.17g\n", fr);
    for (size_t i = 0; i < st.size(); i++) emit(st[i]);
    FILE* g = std::fopen(argv[1], "wb");
    std::fwrite(g_out.data(), sizeof(double), g_out.size(), g);
    std::fclose(g);
    return 0;
}
