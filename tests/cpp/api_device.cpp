// Device part of the C++ API (Proto_B200.H), written like the reference's own tests: the
// "dst |= L(src)" and "dst += L(src)" forms, BoxData algebra, InterpStencil, LevelBoxData exchange
// and the multigrid. Reads inputs from argv[1] (raw float64), writes results to argv[2].
#include <cstdio>
#include <vector>
#include "proto_b200/cpp/Proto_B200.H"

using namespace Proto;

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    const int n = 24;
    std::vector<double> in((size_t)(n + 2) * (n + 2) * (n + 2));
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(in.data(), sizeof(double), in.size(), f) != in.size()) return 3;
    std::fclose(f);
    std::vector<double> out;
    auto emit = [&](const BoxData<double>& b) {
        std::vector<double> h;
        b.copyToHost(h);
        out.insert(out.end(), h.begin(), h.end());
    };
    Box B = Box::Cube(n);
    BoxData<double> u(B.grow(1));
    u.copyFromHost(in);
    auto L = Stencil<double>::Laplacian();
    double h = 1.0 / n;
    // 1. Lu |= L(u, 1/h^2)
    BoxData<double> lu(B);
    lu |= L(u, 1.0 / (h * h));
    emit(lu);
    // 2. lu += L(u) with a user range box, then lu *= 0.5, lu += u (on the intersection)
    lu += L(u, B.grow(-1), 2.0);
    lu *= 0.5;
    lu += u;
    emit(lu);
    // 3. BoxData built from a LazyStencil (inferred range), AvgDown restriction, Constant prolong
    auto A = Stencil<double>::AvgDown(2);
    BoxData<double> c = A(lu);
    emit(c);
    BoxData<double> fine(B, 0.0);
    auto I = InterpStencil<double>::Constant(2);
    I.apply(fine, c, false, 1.0);
    emit(fine);
    // 4. reductions
    std::printf("absMax %.17g sum %.17g max %.17g\n", lu.absMax(), lu.sum(), lu.max());
    // 5. LevelBoxData on a 2x2x2 layout of 12^3 patches, ghost 1, periodic: exchange
    ProblemDomain pd(B, true);
    DisjointBoxLayout layout(pd, Point::Ones(12));
    LevelBoxData<double> lvl(layout, Point::Ones(1));
    for (size_t i = 0; i < lvl.size(); i++) {
        BoxData<double> p = lvl[i];
        p.setVal(0.0);
        BoxData<double> src(const_cast<double*>(u.data()), u.box());
        src.copyTo(p, layout[i]);
    }
    lvl.exchange();
    for (size_t i = 0; i < lvl.size(); i++) emit(lvl[i]);
    // 6. multigrid (archived parameters) on the interior of u as the right-hand side, zero mean
    BoxData<double> rho(B), phi(B, 0.0);
    BoxData<double> usrc(const_cast<double*>(u.data()), u.box());
    usrc.copyTo(rho, B);
    LevelMultigrid mg(n, 3);
    auto hist = mg.solve(rho, phi, 8, 1e-10);
    emit(phi);
    std::printf("mg %zu %.17g %.17g\n", hist.size(), hist.front(), hist.back());
    FILE* g = std::fopen(argv[2], "wb");
    std::fwrite(out.data(), sizeof(double), out.size(), g);
    std::fclose(g);
    return 0;
}
