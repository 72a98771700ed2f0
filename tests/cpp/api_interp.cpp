// InterpStencil<double>::Constant / Linear / Quadratic through the C++ API, one case per run:
//   api_interp kind ratio slo0 slo1 slo2 shi0 shi1 shi2 dlo0 dlo1 dlo2 dhi0 dhi1 dhi2 overwrite scale src dst out
// reads src and dst (raw float64 over their boxes), applies dst |= I(src, scale) (overwrite) or
// dst += I(src, scale), writes dst to out.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "proto_b200/cpp/Proto_B200.H"

using namespace Proto;

static bool read_file(const char* path, std::vector<double>& v)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    const size_t n = std::fread(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
    return n == v.size();
}

int main(int argc, char** argv)
{
    if (argc < 20) return 2;
    int a[14];
    for (int i = 0; i < 14; i++) a[i] = std::atoi(argv[1 + i]);
    const int kind = a[0], ratio = a[1];
    const bool overwrite = std::atoi(argv[15]) != 0;
    const double scale = std::atof(argv[16]);
    Box sb(Point(a[2], a[3], a[4]), Point(a[5], a[6], a[7])), db(Point(a[8], a[9], a[10]), Point(a[11], a[12], a[13]));
    std::vector<double> hs(sb.size()), hd(db.size());
    if (!read_file(argv[17], hs) || !read_file(argv[18], hd)) return 3;
    BoxData<double> src(sb), dst(db);
    src.copyFromHost(hs);
    dst.copyFromHost(hd);
    InterpStencil<double> I = kind == 0 ? InterpStencil<double>::Constant(ratio)
                            : kind == 1 ? InterpStencil<double>::Linear(ratio) : InterpStencil<double>::Quadratic(ratio);
    if (overwrite) dst |= I(src, scale);
    else dst += I(src, scale);
    dst.copyToHost(hd);
    FILE* g = std::fopen(argv[19], "wb");
    std::fwrite(hd.data(), sizeof(double), hd.size(), g);
    std::fclose(g);
    return 0;
}
