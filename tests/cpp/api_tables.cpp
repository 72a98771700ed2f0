// Host-side part of the C++ API (Proto_B200.H): StencilLib tables and Box index math, printed as
// JSON for tests/test_cpp_api.py to compare with the reference's own tables (tests/golden).
#include <cstdio>
#include "proto_b200/cpp/Proto_B200.H"

using namespace Proto;

static void dump(const char* name, const Stencil<double>& S, bool& first)
{
    std::printf("%s\"%s\": {\"coefs\": [", first ? "" : ",\n", name);
    first = false;
    for (size_t j = 0; j < S.size(); j++) std::printf("%s%.17g", j ? ", " : "", S.coefs()[j]);
    std::printf("], \"offs\": [");
    for (size_t j = 0; j < S.size(); j++)
        std::printf("%s[%d, %d, %d]", j ? ", " : "", S.offsets()[j][0], S.offsets()[j][1], S.offsets()[j][2]);
    std::printf("], \"meta\": [%d, %d, %d, %d, %d, %d, %d, %d, %d]}", S.srcRatio()[0], S.srcRatio()[1], S.srcRatio()[2],
                S.destRatio()[0], S.destRatio()[1], S.destRatio()[2], S.destShift()[0], S.destShift()[1],
                S.destShift()[2]);
}

int main()
{
    bool first = true;
    std::printf("{\"stencils\": {\n");
    dump("laplacian", Stencil<double>::Laplacian(), first);
    dump("laplacian19", Stencil<double>::Laplacian_19(), first);
    dump("laplacian27", Stencil<double>::Laplacian_27(), first);
    Stencil<double> L13 = Stencil<double>::Derivative(2, 0, 4);
    for (int d = 1; d < 3; d++) L13 += Stencil<double>::Derivative(2, d, 4);
    dump("laplacian13", L13, first);
    dump("deriv_2_1_4", Stencil<double>::Derivative(2, 1, 4), first);
    dump("deriv_1_2_6", Stencil<double>::Derivative(1, 2, 6), first);
    dump("diffc2f_0_lo_4", Stencil<double>::DiffCellToFace(0, Side::Lo, 4), first);
    dump("diffc2f_2_hi_4", Stencil<double>::DiffCellToFace(2, Side::Hi, 4), first);
    dump("avgdown2", Stencil<double>::AvgDown(2), first);
    dump("sum2", Stencil<double>::Sum(2), first);
    dump("fluxdiv1", Stencil<double>::FluxDivergence(1), first);
    dump("identity", 1.0 * Shift::Zeros(), first);
    std::printf("},\n\"box\": [");
    int cases[4][9] = {{-5, -4, -3, 6, 7, 9, 2, 2, 2}, {-7, 0, 3, -1, 5, 5, 2, 3, 4},
                       {1, -9, -8, 15, -2, 8, 4, 4, 2}, {0, 0, 0, 63, 63, 63, 2, 2, 2}};
    for (int k = 0; k < 4; k++) {
        int* c = cases[k];
        Box b(Point(c[0], c[1], c[2]), Point(c[3], c[4], c[5]));
        Point r(c[6], c[7], c[8]);
        Box co = b.coarsen(r), tc = b.taperCoarsen(r), rf = b.refine(r);
        std::printf("%s{\"coarsen\": [[%d, %d, %d], [%d, %d, %d]], \"taper\": [[%d, %d, %d], [%d, %d, %d]], "
                    "\"refine\": [[%d, %d, %d], [%d, %d, %d]]}",
                    k ? ", " : "", co.low()[0], co.low()[1], co.low()[2], co.high()[0], co.high()[1], co.high()[2],
                    tc.low()[0], tc.low()[1], tc.low()[2], tc.high()[0], tc.high()[1], tc.high()[2], rf.low()[0],
                    rf.low()[1], rf.low()[2], rf.high()[0], rf.high()[1], rf.high()[2]);
    }
    // inferred ranges and index boxes (LazyStencil::inferredRange, Stencil::indexDomain/indexRange)
    auto A = Stencil<double>::AvgDown(2);
    Box src(Point(-4, -4, -4), Point(11, 11, 11));
    Box rg = A.range(src), ir = A.indexRange(src);
    std::printf("],\n\"avg_range\": [[%d, %d, %d], [%d, %d, %d]], \"avg_index_range\": [[%d, %d, %d], [%d, %d, %d]]}\n",
                rg.low()[0], rg.low()[1], rg.low()[2], rg.high()[0], rg.high()[1], rg.high()[2], ir.low()[0],
                ir.low()[1], ir.low()[2], ir.high()[0], ir.high()[1], ir.high()[2]);
    return 0;
}
