// Proto_B200.H — C++ host API with the reference's names and semantics, on the sm_100a library.
//
// Header-only. A C++ caller of the reference's structured-grid path (Proto: Point, Box, Stencil,
// BoxData, InterpStencil, LevelBoxData, the multigrid solver) includes this header instead of
// Proto.H and links libproto_b200.so; data lives on the device and every operation goes through
// the C ABI declared in include/proto_b200.h. Host-side algebra (Box index math, Stencil
// construction, StencilLib builders) is restated here so that coefficient tables, term order and
// index boxes are identical to the reference's (checked against tables dumped from the reference).
//
// Reference files mirrored (paths within the reference project):
//   Point / Box ......... include/base/Proto_Point.H, include/base/implem/Proto_BoxImplem.H
//   Stencil + library ... include/base/Proto_Stencil.H, implem/Proto_StencilImplem.H, implem/Proto_StencilDefs.H
//   BoxData ............. include/base/Proto_BoxData.H, implem/Proto_BoxDataImplem.H
//   InterpStencil ....... include/base/Proto_InterpStencil.H, implem/Proto_InterpStencilDefs.H
//   LevelBoxData ........ include/base/Proto_LevelBoxData.H, Proto_DisjointBoxLayout.H
//   Multigrid ........... include/utils/Proto_LevelMultigridSolver.H,
//                         examples/_archived/LevelMultigrid/src/LevelMultigrid.H
// Errors: the reference aborts (PROTO_ASSERT, MayDay); here a non-zero status throws Proto::Error.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/proto_b200.h"

// Point is usable in device code (the forall kernels of Proto_B200_Forall.cuh) when compiled by nvcc.
#ifdef __CUDACC__
#define PB_HD __host__ __device__
#else
#define PB_HD
#endif

namespace Proto {

enum MemType { HOST = 0, DEVICE = 1 };

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& where)
        : std::runtime_error(where + ": " + pb_status_string(s)), status(s) {}
};
inline void check(int s, const char* where)
{
    if (s != PB_OK) throw Error(s, where);
}

// ---------------------------------------------------------------------------------------------
// Point (3-D). Division rounds toward -infinity (Proto_PointImplem.H:212-239).
// ---------------------------------------------------------------------------------------------
struct Point {
    int v[3] = {0, 0, 0};
    Point() = default;
    PB_HD Point(int x, int y, int z) { v[0] = x; v[1] = y; v[2] = z; }
    PB_HD int& operator[](int d) { return v[d]; }
    PB_HD int operator[](int d) const { return v[d]; }
    PB_HD static Point Zeros() { return Point(0, 0, 0); }
    PB_HD static Point Ones(int s = 1) { return Point(s, s, s); }
    PB_HD static Point Basis(int dir, int s = 1) { Point p; p.v[dir] = s; return p; }
    PB_HD static Point X() { return Basis(0); }
    PB_HD static Point Y() { return Basis(1); }
    PB_HD static Point Z() { return Basis(2); }
    PB_HD Point operator+(const Point& o) const { return Point(v[0] + o[0], v[1] + o[1], v[2] + o[2]); }
    PB_HD Point operator-(const Point& o) const { return Point(v[0] - o[0], v[1] - o[1], v[2] - o[2]); }
    PB_HD Point operator-() const { return Point(-v[0], -v[1], -v[2]); }
    PB_HD Point operator*(const Point& o) const { return Point(v[0] * o[0], v[1] * o[1], v[2] * o[2]); }
    PB_HD Point operator*(int s) const { return Point(v[0] * s, v[1] * s, v[2] * s); }
    PB_HD static int fdiv(int a, int b)
    {
        if (a * b >= 0) return a / b;
        if ((-a) % b == 0) return -(-a / b);
        return -(-a / b + 1);
    }
    PB_HD Point operator/(const Point& o) const { return Point(fdiv(v[0], o[0]), fdiv(v[1], o[1]), fdiv(v[2], o[2])); }
    PB_HD Point operator/(int s) const { return (*this) / Ones(s); }
    PB_HD Point operator%(const Point& o) const { return Point(v[0] % o[0], v[1] % o[1], v[2] % o[2]); }
    PB_HD bool operator==(const Point& o) const { return v[0] == o[0] && v[1] == o[1] && v[2] == o[2]; }
    PB_HD bool operator!=(const Point& o) const { return !(*this == o); }
    PB_HD int sumAbs() const { return (v[0] < 0 ? -v[0] : v[0]) + (v[1] < 0 ? -v[1] : v[1]) + (v[2] < 0 ? -v[2] : v[2]); }
    PB_HD int min() const { return v[0] < v[1] ? (v[0] < v[2] ? v[0] : v[2]) : (v[1] < v[2] ? v[1] : v[2]); }
    PB_HD int max() const { return v[0] > v[1] ? (v[0] > v[2] ? v[0] : v[2]) : (v[1] > v[2] ? v[1] : v[2]); }
};

namespace Side { enum LoHiSide { Lo = 0, Hi = 1 }; }

// ---------------------------------------------------------------------------------------------
// Box: inclusive corners; the default Box is empty (low 0, high -1).
// ---------------------------------------------------------------------------------------------
class Box {
public:
    Box() : m_low(Point::Zeros()), m_high(Point::Ones(-1)) {}
    Box(const Point& lo, const Point& hi) : m_low(lo), m_high(hi) {}
    explicit Box(const Point& size) : m_low(Point::Zeros()), m_high(size - Point::Ones()) {}
    static Box Cube(int n) { return Box(Point::Zeros(), Point::Ones(n - 1)); }
    static Box Kernel(int r) { return Cube(2 * r + 1).shift(Point::Ones(-r)); }
    const Point& low() const { return m_low; }
    const Point& high() const { return m_high; }
    bool empty() const { return m_high[0] < m_low[0] || m_high[1] < m_low[1] || m_high[2] < m_low[2]; }
    int size(int d) const { return empty() ? 0 : m_high[d] - m_low[d] + 1; }
    long long size() const { return empty() ? 0 : (long long)size(0) * size(1) * size(2); }
    Point sizes() const { return Point(size(0), size(1), size(2)); }
    bool containsPoint(const Point& p) const
    {
        for (int d = 0; d < 3; d++)
            if (p[d] < m_low[d] || p[d] > m_high[d]) return false;
        return true;
    }
    bool containsBox(const Box& b) const { return b.empty() || (containsPoint(b.m_low) && containsPoint(b.m_high)); }
    Box shift(const Point& s) const { return Box(m_low + s, m_high + s); }
    Box shift(int dir, int off) const { return shift(Point::Basis(dir, off)); }
    Box grow(int n) const { return grow(Point::Ones(n)); }
    Box grow(const Point& g) const { return Box(m_low - g, m_high + g); }
    Box grow(int dir, int n) const { return grow(Point::Basis(dir, n)); }
    Box grow(int dir, Side::LoHiSide side, int n) const
    {
        return side == Side::Lo ? Box(m_low - Point::Basis(dir, n), m_high) : Box(m_low, m_high + Point::Basis(dir, n));
    }
    Box operator&(const Box& o) const
    {
        Point lo, hi;
        for (int d = 0; d < 3; d++) { lo[d] = std::max(m_low[d], o.m_low[d]); hi[d] = std::min(m_high[d], o.m_high[d]); }
        Box r(lo, hi);
        return r.empty() ? Box() : r;
    }
    void operator&=(const Box& o) { *this = *this & o; }
    // extension to contain a point (Box::operator&(Point), Proto_BoxImplem.H:297-318)
    Box operator&(const Point& p) const
    {
        if (containsPoint(p)) return *this;
        if (empty()) return Box(p, p);
        Point lo, hi;
        for (int d = 0; d < 3; d++) { lo[d] = std::min(m_low[d], p[d]); hi[d] = std::max(m_high[d], p[d]); }
        return Box(lo, hi);
    }
    void operator&=(const Point& p) { *this = *this & p; }
    bool operator==(const Box& o) const { return m_low == o.m_low && m_high == o.m_high; }
    bool operator!=(const Box& o) const { return !(*this == o); }
    // Box::coarsen (Proto_BoxImplem.H:506-553): both corners toward -infinity
    Box coarsen(const Point& r) const { return Box(m_low / r, m_high / r); }
    Box coarsen(int r) const { return coarsen(Point::Ones(r)); }
    Box refine(const Point& r) const { return Box(m_low * r, (m_high + Point::Ones()) * r - Point::Ones()); }
    Box refine(int r) const { return refine(Point::Ones(r)); }
    // Box::taperCoarsen (Proto_BoxImplem.H:555-564): high toward -infinity, low by ceil
    Box taperCoarsen(const Point& r) const
    {
        Point L;
        for (int d = 0; d < 3; d++) L[d] = (int)std::ceil(m_low[d] / (double)r[d]);
        return Box(L, m_high / r);
    }
    bool coarsenable(const Point& r) const { return coarsen(r).refine(r) == *this; }
    Box flatten(int dir, bool upper = false) const
    {
        Point lo = m_low, hi = m_high;
        if (upper) lo[dir] = hi[dir]; else hi[dir] = lo[dir];
        return Box(lo, hi);
    }
    // Box::sindex / index / operator[] (Proto_BoxImplem.H:76-86, 199-225)
    long long index(const Point& p) const
    {
        return (long long)(p[0] - m_low[0]) + (long long)size(0) * ((p[1] - m_low[1]) + (long long)size(1) * (p[2] - m_low[2]));
    }
    Point operator[](long long i) const
    {
        Point p;
        for (int d = 0; d < 3; d++) {
            long long f = size(d);
            p[d] = (int)(i % f) + m_low[d];
            i /= f;
        }
        return p;
    }
    pb_box c() const
    {
        pb_box b;
        for (int d = 0; d < 3; d++) { b.lo[d] = m_low[d]; b.hi[d] = m_high[d]; }
        return b;
    }

private:
    Point m_low, m_high;
};

// ---------------------------------------------------------------------------------------------
// Shift and Stencil<T> (Proto_Stencil.H:66-1001)
// ---------------------------------------------------------------------------------------------
struct Shift {
    Point p;
    explicit Shift(const Point& a) : p(a) {}
    Shift(int x, int y, int z) : p(x, y, z) {}
    static Shift Zeros() { return Shift(Point::Zeros()); }
    static Shift Ones(int s = 1) { return Shift(Point::Ones(s)); }
    static Shift Basis(int dir, int s = 1) { return Shift(Point::Basis(dir, s)); }
    static Shift X(int s = 1) { return Basis(0, s); }
    static Shift Y(int s = 1) { return Basis(1, s); }
    static Shift Z(int s = 1) { return Basis(2, s); }
    const Point& point() const { return p; }
};

template <typename T, unsigned int C, MemType MEM>
class BoxData;
template <typename T, unsigned int C, MemType MEM>
struct LazyStencil;

template <typename T>
class Stencil {
public:
    Stencil() : m_srcRatio(Point::Ones()), m_destRatio(Point::Ones()), m_destShift(Point::Zeros()) {}
    Stencil(Shift s, T coef, Point destRatio = Point::Ones(), Point destShift = Point::Zeros(),
            Point srcRatio = Point::Ones())
        : m_srcRatio(srcRatio), m_destRatio(destRatio), m_destShift(destShift)
    {
        addCoef(coef, s.point());
    }
    // Stencil::addCoef: merge an existing offset, else append (insertion order kept)
    void addCoef(T coef, const Point& off)
    {
        for (size_t j = 0; j < m_offsets.size(); j++)
            if (m_offsets[j] == off) { m_coefs[j] += coef; m_dev.reset(); return; }
        m_coefs.push_back(coef);
        m_offsets.push_back(off);
        m_span &= off;
        m_dev.reset();
    }
    void operator+=(const Stencil& o) { for (size_t j = 0; j < o.m_coefs.size(); j++) addCoef(o.m_coefs[j], o.m_offsets[j]); }
    void operator-=(const Stencil& o) { for (size_t j = 0; j < o.m_coefs.size(); j++) addCoef(-o.m_coefs[j], o.m_offsets[j]); }
    Stencil operator+(const Stencil& o) const { Stencil r = *this; r += o; return r; }
    Stencil operator-(const Stencil& o) const { Stencil r = *this; r -= o; return r; }
    Stencil operator*(T a) const
    {
        Stencil r = *this;
        for (auto& c : r.m_coefs) c *= a;
        r.m_dev.reset();
        return r;
    }
    void operator*=(T a) { for (auto& c : m_coefs) c *= a; m_dev.reset(); }
    // composition (Stencil::operator*(Stencil), Proto_StencilImplem.H:65-81)
    Stencil operator*(const Stencil& o) const
    {
        Stencil r;
        r.m_destRatio = m_destRatio;
        r.m_srcRatio = m_srcRatio;
        r.m_destShift = m_destShift;
        for (size_t i = 0; i < m_coefs.size(); i++)
            for (size_t j = 0; j < o.m_coefs.size(); j++) r.addCoef(m_coefs[i] * o.m_coefs[j], m_offsets[i] + o.m_offsets[j]);
        return r;
    }
    void operator*=(const Stencil& o) { *this = (*this) * o; }
    void invert(int dir)
    {
        for (auto& p : m_offsets) p[dir] = -p[dir];
        recomputeSpan();
    }
    void transpose(int a, int b)
    {
        for (auto& p : m_offsets) std::swap(p[a], p[b]);
        recomputeSpan();
    }
    size_t size() const { return m_coefs.size(); }
    const std::vector<T>& coefs() const { return m_coefs; }
    const std::vector<Point>& offsets() const { return m_offsets; }
    const Box& span() const { return m_span; }
    Point& srcRatio() { m_dev.reset(); return m_srcRatio; }
    const Point& srcRatio() const { return m_srcRatio; }
    Point& destRatio() { m_dev.reset(); return m_destRatio; }
    const Point& destRatio() const { return m_destRatio; }
    Point& destShift() { m_dev.reset(); return m_destShift; }
    const Point& destShift() const { return m_destShift; }
    Point ghost() const
    {
        Point g;
        for (int d = 0; d < 3; d++) g[d] = std::max(std::abs(m_span.low()[d]), std::abs(m_span.high()[d]));
        return g;
    }
    T diagonal() const
    {
        T r = 0;
        for (size_t j = 0; j < m_offsets.size(); j++)
            if (m_offsets[j] == Point::Zeros()) r += m_coefs[j];
        return r;
    }
    // index-space inference (Proto_StencilImplem.H:320-369)
    Box indexRange(const Box& domain) const
    {
        if (domain.empty()) return Box();
        return Box(domain.low() - m_span.low(), domain.high() - m_span.high()).taperCoarsen(m_srcRatio);
    }
    Box indexDomain(const Box& range) const
    {
        if (range.empty()) return Box();
        return range.shift(-m_destShift).taperCoarsen(m_destRatio);
    }
    Box range(const Box& domain) const
    {
        if (domain.empty()) return Box();
        Box r = indexRange(domain);
        return Box(r.low() * m_destRatio, r.high() * m_destRatio).shift(m_destShift);
    }
    Box domain(const Box& range) const
    {
        if (range.empty()) return Box();
        Box d = indexDomain(range);
        d = Box(d.low() * m_srcRatio, d.high() * m_srcRatio);
        return Box(d.low() + m_span.low(), d.high() + m_span.high());
    }

    // device handle (Stencil::closeForDevice): created on first use, immutable afterwards
    const pb_stencil* device() const
    {
        if (!m_dev) {
            std::vector<double> c(m_coefs.begin(), m_coefs.end());
            std::vector<int> o;
            for (auto& p : m_offsets) { o.push_back(p[0]); o.push_back(p[1]); o.push_back(p[2]); }
            pb_stencil* h = nullptr;
            check(pb_stencil_create(c.data(), o.data(), (int)c.size(), m_srcRatio.v, m_destRatio.v, m_destShift.v, &h),
                  "Stencil::closeForDevice");
            m_dev = std::shared_ptr<pb_stencil>(h, [](pb_stencil* s) { pb_stencil_destroy(s); });
        }
        return m_dev.get();
    }

    // Stencil::apply (Proto_StencilImplem.H:412-431); an empty box is inferred on the device side
    template <unsigned int C>
    void apply(const BoxData<T, C, DEVICE>& src, BoxData<T, C, DEVICE>& dst, const Box& box, bool initToZero,
               T scale = 1) const;
    template <unsigned int C>
    LazyStencil<T, C, DEVICE> operator()(const BoxData<T, C, DEVICE>& src, T scale = 1) const
    {
        return LazyStencil<T, C, DEVICE>{this, &src, Box(), scale};
    }
    template <unsigned int C>
    LazyStencil<T, C, DEVICE> operator()(const BoxData<T, C, DEVICE>& src, Box range, T scale = 1) const
    {
        return LazyStencil<T, C, DEVICE>{this, &src, range, scale};
    }

    // ---- StencilLib (Proto_StencilDefs.H) ----
    static Stencil Laplacian()
    {
        Stencil r = ((T)(-6)) * Shift::Zeros();
        for (int d = 0; d < 3; d++) {
            r += ((T)1) * Shift::Basis(d, 1);
            r += ((T)1) * Shift::Basis(d, -1);
        }
        return r;
    }
    static Stencil Laplacian_19()
    {
        Stencil r = ((T)(-24.0)) * Shift::Zeros();
        Box K = Box::Kernel(1);
        for (long long i = 0; i < K.size(); i++) {
            Point p = K[i];
            int s = p.sumAbs();
            if (s == 1) r += ((T)2.0) * Shift(p);
            else if (s == 2) r += ((T)1.0) * Shift(p);
        }
        r *= (T)(1.0 / 6.0);
        return r;
    }
    static Stencil Laplacian_27()
    {
        Stencil r = ((T)(-64.0 / 15.0)) * Shift::Zeros();
        Box K = Box::Kernel(1);
        for (long long i = 0; i < K.size(); i++) {
            Point p = K[i];
            int s = p.sumAbs();
            if (s == 1) r += ((T)(7.0 / 15.0)) * Shift(p);
            else if (s == 2) r += ((T)(1.0 / 10.0)) * Shift(p);
            else if (s == 3) r += ((T)(1.0 / 30.0)) * Shift(p);
        }
        return r;
    }
    // n-th derivative in direction dir to the given (even-rounded) order: the standard central
    // difference correction series in powers of the second difference (published expansions of
    // h^n D^n in delta^2; the same tables as Proto_StencilDefs.H:393-457)
    static Stencil Derivative(int n, int dir, int order = 2)
    {
        const int M = 6;
        if (order % 2 != 0) order++;
        Point e = Point::Basis(dir);
        Stencil factor = ((T)1.0) * Shift(e) + ((T)(-2.0)) * Shift::Zeros() + ((T)1.0) * Shift(e * (-1));
        Stencil temps[M];
        Stencil deriv;
        if (n % 2 == 0) {
            const T even[M][M] = {{1., -1. / 12, 1. / 90, -1. / 560, 1. / 3150, -1. / 16632},
                                  {0, 1., -1. / 6, 7. / 240, -41. / 7560, 479. / 453600},
                                  {0, 0, 1., -1. / 4, 13. / 240, -139. / 12096},
                                  {0, 0, 0, 1., -1. / 3, 31. / 360},
                                  {0, 0, 0, 0, 1., -5. / 12},
                                  {0, 0, 0, 0, 0, 1.}};
            int p = (n - 2) / 2;
            temps[0] = factor;
            for (int k = 1; k < M; k++) temps[k] = temps[k - 1] * factor;
            for (int k = 0; k < (n + order - 2) / 2; k++) deriv += temps[k] * even[p][k];
        } else {
            const T odd[M][M] = {{1., -1. / 6, 1. / 30, -1. / 140, 1. / 630, -1. / 2772},
                                 {0, 1., -1. / 4, 7. / 120, -41. / 3024, 479. / 151200},
                                 {0, 0, 1., -1. / 3, 13. / 144, -139. / 6048},
                                 {0, 0, 0, 1., -5. / 12, 31. / 240},
                                 {0, 0, 0, 0, 1., -1. / 2},
                                 {0, 0, 0, 0, 0, 1.}};
            int p = (n - 1) / 2;
            temps[0] = ((T)0.5) * Shift(e) + ((T)(-0.5)) * Shift(e * (-1));
            for (int k = 1; k < M; k++) temps[k] = temps[k - 1] * factor;
            for (int k = 0; k < (n + 1 + order - 2) / 2; k++) deriv += temps[k] * odd[p][k];
        }
        return deriv;
    }
    static Stencil AvgDown(const Point& r)
    {
        Stencil s;
        Box k(r);
        T c = 1.0 / k.size();
        for (long long i = 0; i < k.size(); i++) s += c * Shift(k[i]);
        s.m_srcRatio = r;
        return s;
    }
    static Stencil AvgDown(int r) { return AvgDown(Point::Ones(r)); }
    static Stencil Sum(const Point& r)
    {
        Stencil s;
        Box k(r);
        T c = 1.0;
        for (long long i = 0; i < k.size(); i++) s += c * Shift(k[i]);
        s.m_srcRatio = r;
        return s;
    }
    static Stencil Sum(int r) { return Sum(Point::Ones(r)); }
    static Stencil DiffCellToFace(int dir, Side::LoHiSide side = Side::Lo, int order = 4)
    {
        Stencil r;
        if (order == 4) {
            T c[4] = {1, -15, 15, -1};
            r = c[0] * Shift::Basis(dir, -2) + c[1] * Shift::Basis(dir, -1) + c[2] * Shift::Zeros() + c[3] * Shift::Basis(dir, 1);
            r *= (T)(1.0 / 12.0);
        } else if (order == 2) {
            r = ((T)(-1.0)) * Shift::Basis(dir, -1) + ((T)1.0) * Shift::Zeros();
        } else {
            throw Error(PB_ERR_UNSUPPORTED, "Stencil::DiffCellToFace order");
        }
        if (side == Side::Hi) r.invert(dir);
        return r;
    }
    static Stencil FluxDivergence(int dir)
    {
        return ((T)(-1)) * Shift::Zeros() + ((T)(1.0)) * Shift::Basis(dir);
    }

private:
    void recomputeSpan()
    {
        m_span = Box();
        for (auto& p : m_offsets) m_span &= p;
        m_dev.reset();
    }
    std::vector<T> m_coefs;
    std::vector<Point> m_offsets;
    Point m_srcRatio, m_destRatio, m_destShift;
    Box m_span;
    mutable std::shared_ptr<pb_stencil> m_dev;
};

template <typename T>
inline Stencil<T> operator*(T c, Shift s) { return Stencil<T>(s, c); }
inline Stencil<double> operator*(int c, Shift s) { return Stencil<double>(s, (double)c); }
template <typename T>
inline Stencil<T> operator*(T c, const Stencil<T>& s) { return s * c; }
template <typename T>
inline Stencil<T> operator-(const Stencil<T>& s) { return s * (T)(-1); }

// ---------------------------------------------------------------------------------------------
// BoxData<T, C, DEVICE>: C components on a Box, component-major, x fastest, in device memory.
// ---------------------------------------------------------------------------------------------
template <typename T, unsigned int C = 1, MemType MEM = DEVICE>
class BoxData {
    static_assert(MEM == DEVICE, "Proto_B200.H holds BoxData in device memory only");

public:
    BoxData() = default;
    explicit BoxData(const Box& b) { define(b); }
    BoxData(const Box& b, T init) { define(b); setVal(init); }
    // alias of caller-owned device memory (BoxData(const T*, const Box&, int))
    BoxData(T* ptr, const Box& b, int ncomp = C) : m_box(b), m_ptr(ptr) { (void)ncomp; }
    BoxData(LazyStencil<T, C, DEVICE>&& op);
    BoxData(BoxData&&) = default;
    BoxData& operator=(BoxData&&) = default;
    BoxData(const BoxData&) = delete;

    void define(const Box& b)
    {
        m_box = b;
        size_t bytes = sizeof(T) * (size_t)std::max<long long>(1, b.size()) * C;
        T* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); throw Error(PB_ERR_NOMEM, "BoxData::define"); }
        m_owner = std::shared_ptr<T>(p, [](T* q) { cudaFree(q); });
        m_ptr = p;
    }
    const Box& box() const { return m_box; }
    T* data(unsigned int c = 0) { return m_ptr + (size_t)c * m_box.size(); }
    const T* data(unsigned int c = 0) const { return m_ptr + (size_t)c * m_box.size(); }
    size_t size() const { return (size_t)m_box.size() * C; }
    bool defined() const { return m_ptr != nullptr; }

    // host transfers (synchronous, like proto_memcpy)
    void copyToHost(std::vector<T>& out) const
    {
        out.resize(size());
        check(cudaMemcpy(out.data(), m_ptr, size() * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : PB_ERR_CUDA,
              "BoxData::copyToHost");
    }
    void copyFromHost(const std::vector<T>& in)
    {
        check(in.size() == size() && cudaMemcpy(m_ptr, in.data(), size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess
                  ? 0 : PB_ERR_CUDA, "BoxData::copyFromHost");
    }

    void setVal(T v, cudaStream_t st = 0) { check(pb_boxdata_scalar_f64(PB_OP_ASSIGN, dp(), m_box.c(), Box().c(), v, C, st), "BoxData::setVal"); }
    void setToZero(cudaStream_t st = 0) { setVal(0, st); }
    BoxData& operator+=(const BoxData& o) { return binop(PB_OP_ADD, o); }
    BoxData& operator-=(const BoxData& o) { return binop(PB_OP_SUB, o); }
    BoxData& operator*=(const BoxData& o) { return binop(PB_OP_MUL, o); }
    BoxData& operator/=(const BoxData& o) { return binop(PB_OP_DIV, o); }
    BoxData& operator+=(T s) { return scalar(PB_OP_ADD, s); }
    BoxData& operator-=(T s) { return scalar(PB_OP_SUB, s); }
    BoxData& operator*=(T s) { return scalar(PB_OP_MUL, s); }
    BoxData& operator/=(T s) { return scalar(PB_OP_DIV, s); }
    void copyTo(BoxData& dst) const { copyTo(dst, m_box, Point::Zeros()); }
    void copyTo(BoxData& dst, const Box& srcBox, const Point& shift = Point::Zeros()) const
    {
        check(pb_boxdata_copy_f64(dp(), m_box.c(), dst.dp(), dst.m_box.c(), srcBox.c(), shift.v, C, 0), "BoxData::copyTo");
    }
    T reduce(int op) const
    {
        static_assert(C == 1, "reductions over one component");
        double r = 0;
        check(pb_reduce_f64(op, dp(), m_box.c(), Box().c(), &r, 0), "BoxData::reduce");
        return (T)r;
    }
    T absMax() const { return reduce(2); }
    T max() const { return reduce(0); }
    T min() const { return reduce(1); }
    T sum() const { return reduce(3); }
    T sumAbs() const { return reduce(4); }
    T sumSquare() const { return reduce(5); }

    double* dp() const { return reinterpret_cast<double*>(m_ptr); }

private:
    BoxData& binop(int op, const BoxData& o)
    {
        check(pb_boxdata_op_f64(op, dp(), m_box.c(), o.dp(), o.m_box.c(), C, 0), "BoxData::operatorT");
        return *this;
    }
    BoxData& scalar(int op, T s)
    {
        check(pb_boxdata_scalar_f64(op, dp(), m_box.c(), Box().c(), (double)s, C, 0), "BoxData::operator(scalar)");
        return *this;
    }
    Box m_box;
    std::shared_ptr<T> m_owner;
    T* m_ptr = nullptr;
};

template <typename T, unsigned int C, MemType MEM>
struct LazyStencil {
    const Stencil<T>* stencil;
    const BoxData<T, C, MEM>* src;
    Box range;
    T scale;
    Box inferredRange() const { return stencil->range(src->box()); }
    void apply(BoxData<T, C, MEM>& dst, bool overwrite) const
    {
        stencil->apply(*src, dst, range.empty() ? Box() : stencil->indexDomain(range), overwrite, scale);
    }
};

template <typename T>
template <unsigned int C>
void Stencil<T>::apply(const BoxData<T, C, DEVICE>& src, BoxData<T, C, DEVICE>& dst, const Box& box, bool initToZero,
                       T scale) const
{
    if (m_coefs.empty()) return;
    int s;
    if (sizeof(T) == 8)
        s = pb_stencil_apply_f64(device(), (const double*)src.data(), src.box().c(), (double*)dst.data(), dst.box().c(),
                                 box.c(), C, initToZero, (double)scale, 0);
    else
        s = pb_stencil_apply_f32(device(), (const float*)src.data(), src.box().c(), (float*)dst.data(), dst.box().c(),
                                 box.c(), C, initToZero, (float)scale, 0);
    check(s, "Stencil::apply");
}

template <typename T, unsigned int C, MemType MEM>
BoxData<T, C, MEM>::BoxData(LazyStencil<T, C, DEVICE>&& op)
{
    Box r = op.range.empty() ? op.inferredRange() : op.range;
    define(r);
    op.apply(*this, true);
}

template <typename T, unsigned int C>
BoxData<T, C, DEVICE>& operator|=(BoxData<T, C, DEVICE>& dst, LazyStencil<T, C, DEVICE>&& op)
{
    op.apply(dst, true);
    return dst;
}
template <typename T, unsigned int C>
BoxData<T, C, DEVICE>& operator+=(BoxData<T, C, DEVICE>& dst, LazyStencil<T, C, DEVICE>&& op)
{
    op.apply(dst, false);
    return dst;
}

// Fused stencil + pointwise update in one pass (what "BoxData Lu = L(u, s); forall(...)" computes):
//   out = a*L(u, s) + b*u   or   out = u + a*L(u, s)
template <typename T>
void applyFused(const Stencil<T>& L, int epilogue, const BoxData<T, 1, DEVICE>& u, BoxData<T, 1, DEVICE>& out, T scale,
                T a, T b = 0)
{
    check(pb_stencil_apply_fused_f64(L.device(), epilogue, u.dp(), u.box().c(), out.dp(), out.box().c(), Box().c(),
                                     scale, a, b, 0),
          "applyFused");
}

// ---------------------------------------------------------------------------------------------
// InterpStencil<T>::Constant (piecewise-constant prolongation)
// ---------------------------------------------------------------------------------------------
template <typename T>
class InterpStencil {
public:
    enum Kind { CONSTANT = 0, LINEAR = 1, QUADRATIC = 2 };
    InterpStencil() = default;
    // InterpStencil<T>::Constant / Linear / Quadratic (Proto_InterpStencilDefs.H:1-80): per
    // direction, one dest-refined 1-D stencil per fine offset s < r
    static InterpStencil Constant(int r) { return Constant(Point::Ones(r)); }
    static InterpStencil Constant(const Point& r)
    {
        return build(CONSTANT, r, [](int, int, int) { return Stencil<T>(Shift::Zeros(), (T)1.0); });
    }
    static InterpStencil Linear(int r) { return Linear(Point::Ones(r)); }
    static InterpStencil Linear(const Point& r)
    {
        return build(LINEAR, r, [](int dir, int shift, int rr) {
            const double rd = rr, sd = shift;
            const double p = sd / rd, q = (rd - sd) / rd;
            return Stencil<T>(Shift::Zeros(), (T)q) + Stencil<T>(Shift::Basis(dir, 1), (T)p);
        });
    }
    static InterpStencil Quadratic(int r) { return Quadratic(Point::Ones(r)); }
    static InterpStencil Quadratic(const Point& r)
    {
        return build(QUADRATIC, r, [](int dir, int shift, int rr) {
            Stencil<T> S;
            for (int ii = -1; ii <= 1; ii++) S += Stencil<T>(Shift::Basis(dir, ii), (T)qcoef(shift, rr, ii));
            return S;
        });
    }
    int ratio() const { return m_ratio[0]; }
    const Point& ratioPoint() const { return m_ratio; }
    Kind kind() const { return m_kind; }
    // InterpStencil::range (Proto_InterpStencilImplem.H:35-53): the bounding box over the shifts
    Box range(const Box& src) const
    {
        Point L, H;
        for (int d = 0; d < 3; d++)
            for (size_t s = 0; s < m_interp[d].size(); s++) {
                Box di = m_interp[d][s].range(src);
                if (s == 0) { L[d] = di.low()[d]; H[d] = di.high()[d]; }
                else { L[d] = std::min(di.low()[d], L[d]); H[d] = std::max(di.high()[d], H[d]); }
            }
        return Box(L, H);
    }
    struct Lazy {
        const InterpStencil* op;
        const BoxData<T, 1, DEVICE>* src;
        T scale;
    };
    Lazy operator()(const BoxData<T, 1, DEVICE>& src, T scale = 1) const { return Lazy{this, &src, scale}; }
    // InterpStencil::apply (Proto_InterpStencilImplem.H:83-112): the 1-D stages in x, y, z, then
    // dst (|= or +=) scale * stage on range(src) & dst (or the given range). Constant with one ratio
    // takes a single fused kernel, bitwise the staged result.
    void apply(BoxData<T, 1, DEVICE>& dst, const BoxData<T, 1, DEVICE>& src, bool overwrite, T scale,
               Box rangeBox = Box()) const
    {
        const bool iso = m_ratio[0] == m_ratio[1] && m_ratio[1] == m_ratio[2];
        if (m_kind == CONSTANT && iso && rangeBox.empty()) {
            check(pb_interp_constant_f64(m_ratio[0], src.dp(), src.box().c(), dst.dp(), dst.box().c(), overwrite, scale, 0),
                  "InterpStencil::apply");
            return;
        }
        if (rangeBox.empty()) rangeBox = range(src.box()) & dst.box();
        BoxData<T, 1, DEVICE> s0 = stage(m_interp[0], src);
        BoxData<T, 1, DEVICE> s1 = stage(m_interp[1], s0);
        BoxData<T, 1, DEVICE> s2 = stage(m_interp[2], s1);
        Stencil<T> S(Shift::Zeros(), scale);
        S.apply(s2, dst, rangeBox, overwrite, (T)1);
    }

private:
    // qcoef of Proto_InterpStencilDefs.H:40-58 (the quadratic weights)
    static double qcoef(int a_ni, int a_r, int a_side)
    {
        double n = a_ni, r = a_r, coef = 0;
        if (a_side == -1) coef = 1.0 + 3.0 * n + 3.0 * n * n - 3.0 * r - 6.0 * n * r + 2.0 * r * r;
        else if (a_side == 0) coef = -2.0 - 6.0 * n - 6.0 * n * n + 3.0 * r + 6.0 * n * r + 5.0 * r * r;
        else if (a_side == 1) coef = -(-1.0 - 3.0 * n - 3.0 * n * n + r * r);
        coef /= (6.0 * r * r);
        return coef;
    }
    template <class F>
    static InterpStencil build(Kind kind, const Point& r, F make)
    {
        if (r.min() <= 0) throw Error(PB_ERR_ARG, "InterpStencil: non-positive refinement ratio");
        InterpStencil I;
        I.m_kind = kind;
        I.m_ratio = r;
        for (int d = 0; d < 3; d++)
            for (int sft = 0; sft < r[d]; sft++) {
                Stencil<T> S = make(d, sft, r[d]);
                Point ratio = Point::Ones();
                ratio[d] = r[d];
                S.destRatio() = ratio;
                S.destShift() = Point::Basis(d, sft);
                I.m_interp[d].push_back(S);
            }
        return I;
    }
    // InterpStencil1D applied as a LazyStencil into a new BoxData (Proto_InterpStencil1DImplem.H:88-118):
    // the output covers the bounding box of the shifts' ranges, each shift fills its own cells
    static BoxData<T, 1, DEVICE> stage(const std::vector<Stencil<T>>& S, const BoxData<T, 1, DEVICE>& src)
    {
        Box R;
        for (size_t s = 0; s < S.size(); s++) {
            Box r = S[s].range(src.box());
            R = (s == 0) ? r : ((R & r.low()) & r.high());
        }
        BoxData<T, 1, DEVICE> out(R);
        for (size_t s = 0; s < S.size(); s++) {
            Box b(src.box().low() - S[s].span().low(), src.box().high() - S[s].span().high());
            S[s].apply(src, out, b.taperCoarsen(S[s].srcRatio()), true, (T)1);
        }
        return out;
    }
    Kind m_kind = CONSTANT;
    Point m_ratio = Point::Ones(2);
    std::vector<Stencil<T>> m_interp[3];
};
template <typename T>
BoxData<T, 1, DEVICE>& operator|=(BoxData<T, 1, DEVICE>& dst, typename InterpStencil<T>::Lazy&& op)
{
    op.op->apply(dst, *op.src, true, op.scale);
    return dst;
}
template <typename T>
BoxData<T, 1, DEVICE>& operator+=(BoxData<T, 1, DEVICE>& dst, typename InterpStencil<T>::Lazy&& op)
{
    op.op->apply(dst, *op.src, false, op.scale);
    return dst;
}

// ---------------------------------------------------------------------------------------------
// ProblemDomain, DisjointBoxLayout (any disjoint tiling) and LevelBoxData<double,1,DEVICE>
// ---------------------------------------------------------------------------------------------
struct ProblemDomain {
    Box box;
    std::array<bool, 3> periodic{{true, true, true}};
    ProblemDomain() = default;
    ProblemDomain(const Box& b, bool per) : box(b) { periodic.fill(per); }
    ProblemDomain(const Box& b, const std::array<bool, 3>& per) : box(b), periodic(per) {}
    bool isPeriodic(int d) const { return periodic[d]; }
};

class DisjointBoxLayout {
public:
    DisjointBoxLayout() = default;
    // fixed box size (the reference's layout)
    DisjointBoxLayout(const ProblemDomain& pd, const Point& boxSize) : m_domain(pd)
    {
        Box cb = pd.box.coarsen(boxSize);
        for (long long i = 0; i < cb.size(); i++) {
            Point p = cb[i];
            m_boxes.push_back(Box(p * boxSize, (p + Point::Ones()) * boxSize - Point::Ones()));
        }
    }
    // any disjoint tiling of the domain (uneven patch sizes)
    DisjointBoxLayout(const ProblemDomain& pd, const std::vector<Box>& boxes) : m_domain(pd), m_boxes(boxes) {}
    const ProblemDomain& domain() const { return m_domain; }
    size_t size() const { return m_boxes.size(); }
    const Box& operator[](size_t i) const { return m_boxes[i]; }
    const std::vector<Box>& boxes() const { return m_boxes; }

private:
    ProblemDomain m_domain;
    std::vector<Box> m_boxes;
};

template <typename T = double, unsigned int C = 1, MemType MEM = DEVICE>
class LevelBoxData {
    static_assert(C == 1 && MEM == DEVICE, "Proto_B200.H levels hold one device component");

public:
    LevelBoxData() = default;
    LevelBoxData(const DisjointBoxLayout& layout, const Point& ghost) { define(layout, ghost); }
    void define(const DisjointBoxLayout& layout, const Point& ghost)
    {
        m_layout = layout;
        m_ghost = ghost;
        std::vector<pb_box> bx;
        for (auto& b : layout.boxes()) bx.push_back(b.c());
        int per[3] = {layout.domain().periodic[0], layout.domain().periodic[1], layout.domain().periodic[2]};
        pb_level* lv = nullptr;
        check(pb_level_create(bx.data(), (int)bx.size(), ghost.v, layout.domain().box.c(), per, 1, &lv), "LevelBoxData::define");
        m_level = std::shared_ptr<pb_level>(lv, [](pb_level* l) { pb_level_destroy(l); });
        m_offsets.resize(bx.size());
        long long slab = 0;
        check(pb_level_layout(lv, m_offsets.data(), &slab, nullptr), "LevelBoxData::define");
        m_slab = BoxData<T, 1, DEVICE>(Box(Point(0, 0, 0), Point((int)std::max<long long>(slab, 1) - 1, 0, 0)));
    }
    const DisjointBoxLayout& layout() const { return m_layout; }
    Point ghost() const { return m_ghost; }
    size_t size() const { return m_layout.size(); }
    // patch i as an alias into the level's slab, on its box grown by the ghost width
    BoxData<T, 1, DEVICE> operator[](size_t i) const
    {
        return BoxData<T, 1, DEVICE>(const_cast<T*>(m_slab.data()) + m_offsets[i], m_layout[i].grow(m_ghost));
    }
    void exchange(cudaStream_t st = 0) { check(pb_level_exchange_f64(m_level.get(), m_slab.dp(), st), "LevelBoxData::exchange"); }
    void setToZero() { m_slab.setVal(0); }
    T* slab() { return m_slab.data(); }
    pb_level* handle() const { return m_level.get(); }
    T absMax() const
    {
        double m = 0;
        for (size_t i = 0; i < size(); i++) {
            double r = 0;
            auto p = (*this)[i];
            check(pb_reduce_f64(2, p.dp(), p.box().c(), m_layout[i].c(), &r, 0), "LevelBoxData::absMax");
            m = std::max(m, r);
        }
        return (T)m;
    }

private:
    DisjointBoxLayout m_layout;
    Point m_ghost;
    std::shared_ptr<pb_level> m_level;
    std::vector<long long> m_offsets;
    BoxData<T, 1, DEVICE> m_slab;
};

// ---------------------------------------------------------------------------------------------
// Multigrid: periodic point-Jacobi V-cycles on one grid (LevelMultigrid / LevelMultigridSolver)
// ---------------------------------------------------------------------------------------------
class LevelMultigrid {
public:
    // the archived solver's signature (examples/_archived/LevelMultigrid/src/LevelMultigrid.H:15):
    // a periodic cube domain [0, n-1]^3 tiled by any layout, dx = 1/n, numLevels coarsenings; V(6,6),
    // point Jacobi with weight 1/(4 DIM) (omega = 0.5), 10 bottom sweeps
    LevelMultigrid(const DisjointBoxLayout& layout, double dx, int numLevels) : LevelMultigrid(cube_edge(layout, dx), numLevels)
    {
        m_layout = layout;
    }
    void define(const DisjointBoxLayout& layout, double dx, int numLevels) { *this = LevelMultigrid(layout, dx, numLevels); }
    // one V-cycle on phi for right-hand side rhs (LevelMultigrid::vCycle, LevelMultigrid.cpp:133-158)
    void vCycle(LevelBoxData<double>& phi, LevelBoxData<double>& rhs) { cycles(phi, rhs, 1); }
    // max-norm residual of phi (LevelMultigrid::resnorm, LevelMultigrid.cpp:71-88)
    double resnorm(LevelBoxData<double>& phi, LevelBoxData<double>& rhs) { return cycles(phi, rhs, 0); }

    // n: finest edge; numLevels: coarsenings (the archived driver's numLevels argument)
    LevelMultigrid(int n, int numLevels, int nu1 = 2 * 3, int nu2 = 2 * 3, int nuBottom = 10, double omega = 0.5)
    {
        pb_mg_params p{};
        p.n = n;
        p.levels = numLevels;
        p.nu1 = nu1;
        p.nu2 = nu2;
        p.nu_bottom = nuBottom;
        p.omega = omega;
        p.beta = 1.0;
        p.form = PB_MG_POISSON;
        p.precision = PB_MG_FP64;
        p.max_iter = 100;
        p.tol = 1e-10;
        m_p = p;
        pb_mg* h = nullptr;
        check(pb_mg_create(&m_p, &h), "LevelMultigrid");
        m_h = std::shared_ptr<pb_mg>(h, [](pb_mg* m) { pb_mg_destroy(m); });
    }
    // solves L_h phi = rho from the given phi; returns the residual history
    std::vector<double> solve(const BoxData<double, 1, DEVICE>& rho, BoxData<double, 1, DEVICE>& phi, int maxIter,
                              double tol)
    {
        m_p.max_iter = maxIter;
        m_p.tol = tol;
        m_h.reset();                // parameters changed: rebuild (cheap relative to a solve)
        pb_mg* h = nullptr;
        check(pb_mg_create(&m_p, &h), "LevelMultigrid::solve");
        m_h = std::shared_ptr<pb_mg>(h, [](pb_mg* m) { pb_mg_destroy(m); });
        std::vector<double> hist(maxIter + 1);
        int it = 0;
        check(pb_mg_solve(m_h.get(), rho.dp(), phi.dp(), &it, hist.data(), 0), "LevelMultigrid::solve");
        hist.resize(it + 1);
        return hist;
    }

private:
    static int cube_edge(const DisjointBoxLayout& layout, double dx)
    {
        const Box& d = layout.domain().box;
        const int n = d.size(0);
        if (d.low() != Point::Zeros() || d.size(1) != n || d.size(2) != n || !layout.domain().periodic[0] ||
            !layout.domain().periodic[1] || !layout.domain().periodic[2] || dx != 1.0 / n)
            throw Error(PB_ERR_UNSUPPORTED, "LevelMultigrid: periodic cube [0,n-1]^3 with dx = 1/n expected");
        return n;
    }
    // gathers the valid cells of phi and rhs into the solver's n^3 arrays, runs k cycles (0: the
    // norm only), scatters phi back and refreshes its ghosts; returns the last residual norm
    double cycles(LevelBoxData<double>& phi, LevelBoxData<double>& rhs, int k)
    {
        const Box dom = m_layout.domain().box;
        if (!m_full) {
            m_full = std::make_shared<BoxData<double, 1, DEVICE>>(dom);
            m_rhs = std::make_shared<BoxData<double, 1, DEVICE>>(dom);
        }
        for (size_t i = 0; i < phi.size(); i++) {
            phi[i].copyTo(*m_full, m_layout[i]);
            rhs[i].copyTo(*m_rhs, m_layout[i]);
        }
        std::vector<double> hist(k + 1);
        int it = 0;
        check(pb_mg_solve_n(m_h.get(), m_rhs->dp(), m_full->dp(), k, 0.0, &it, hist.data(), 0), "LevelMultigrid::vCycle");
        for (size_t i = 0; i < phi.size(); i++) {
            BoxData<double> p = phi[i];
            m_full->copyTo(p, m_layout[i]);
        }
        phi.exchange();
        return hist[it];
    }
    pb_mg_params m_p;
    std::shared_ptr<pb_mg> m_h;
    DisjointBoxLayout m_layout;
    std::shared_ptr<BoxData<double, 1, DEVICE>> m_full, m_rhs;
};

// ---------------------------------------------------------------------------------------------
// BoxOp_Laplace (examples/_common/BoxOp_Laplace.H through BoxOp::operator(),
// include/base/implem/Proto_BoxOpImplem.H:130-175): the 4th-order flux-form Laplacian
//   L(phi) = fluxScale * sum_d DIV_d(DiffCellToFace(d, Lo, 4)(phi) / dx) / dx   (* scale)
// applied on the device, bitwise the reference's operator. Any class with the same
// operator()(output, state, scale) can stand in for it in LevelOp (a plugged-in operator).
// ---------------------------------------------------------------------------------------------
template <typename T = double, MemType MEM = DEVICE>
class BoxOp_Laplace {
    static_assert(std::is_same<T, double>::value && MEM == DEVICE, "BoxOp_Laplace<double, DEVICE>");

public:
    static constexpr unsigned int numState() { return 1; }
    static constexpr unsigned int numAux() { return 0; }
    static constexpr int order() { return 4; }
    static Point ghost() { return Point::Ones(2); }
    static Point auxGhost() { return Point::Zeros(); }
    BoxOp_Laplace() = default;
    explicit BoxOp_Laplace(double dx) { define(dx); }
    void define(double dx) { m_dx = dx; }
    // BoxOp::define(layout, index, dx): the operator keeps dx
    void define(const DisjointBoxLayout&, size_t, double dx) { define(dx); }
    double dx() const { return m_dx; }
    double dxMin() const { return m_dx; }
    double spectralRadius() const { return (2.0 * 3) / (m_dx * m_dx); }
    void setFluxScale(T s) { m_fluxScale = s; }
    T fluxScale() const { return m_fluxScale; }
    // output |= L(state) on output's box (state must cover it grown by ghost())
    void operator()(BoxData<T, 1, DEVICE>& output, const BoxData<T, 1, DEVICE>& state, T scale = 1.0) const
    {
        check(pb_boxop_laplace_f64(state.dp(), state.box().c(), output.dp(), output.box().c(), Box().c(), m_dx,
                                   m_fluxScale, scale, 0), "BoxOp_Laplace::operator()");
    }
    // out of place on a range box
    BoxData<T, 1, DEVICE> operator()(const BoxData<T, 1, DEVICE>& state, Box range, T scale = 1.0) const
    {
        BoxData<T, 1, DEVICE> out(range);
        (*this)(out, state, scale);
        return out;
    }

private:
    double m_dx = 1.0;
    T m_fluxScale = 1.0;
};

// ---------------------------------------------------------------------------------------------
// LevelOp<OpType>: the operator of every patch of a level (include/base/Proto_LevelOp.H:25-116):
// exchange the state's ghost cells, then OpType::operator()(output[i], state[i], scale) per patch.
// OpType is BoxOp_Laplace or any class with define(dx), operator()(BoxData&, const BoxData&, T)
// and spectralRadius().
// ---------------------------------------------------------------------------------------------
template <template <typename, MemType> class OpType, typename T = double, MemType MEM = DEVICE>
class LevelOp {
public:
    LevelOp() = default;
    LevelOp(const DisjointBoxLayout& layout, T dx) { define(layout, dx); }
    void define(const DisjointBoxLayout& layout, T dx)
    {
        m_layout = layout;
        m_ops.assign(layout.size(), OpType<T, MEM>());
        for (auto& op : m_ops) op.define(dx);
    }
    const OpType<T, MEM>& operator[](size_t i) const { return m_ops[i]; }
    OpType<T, MEM>& operator[](size_t i) { return m_ops[i]; }
    double spectralRadius() const { return m_ops.empty() ? 0.0 : m_ops[0].spectralRadius(); }
    const DisjointBoxLayout& layout() const { return m_layout; }
    void operator()(LevelBoxData<T>& output, LevelBoxData<T>& state, T scale = 1.0) const
    {
        state.exchange();
        for (size_t i = 0; i < m_layout.size(); i++) {
            BoxData<T> in = state[i];
            BoxData<T> whole = output[i];
            apply_valid(m_ops[i], whole, in, m_layout[i], scale);
        }
    }

private:
    // the operator on the valid box of a patch whose output field carries ghost cells: evaluate
    // into a valid-box temporary and copy it in
    static void apply_valid(const OpType<T, MEM>& op, BoxData<T>& out_grown, const BoxData<T>& in, const Box& valid,
                            T scale)
    {
        if (out_grown.box() == valid) {
            op(out_grown, in, scale);
            return;
        }
        BoxData<T> tmp(valid);
        op(tmp, in, scale);
        tmp.copyTo(out_grown, valid);
    }
    DisjointBoxLayout m_layout;
    std::vector<OpType<T, MEM>> m_ops;
};

// ---------------------------------------------------------------------------------------------
// LevelMultigridSolver<BoxOp_Laplace, double> with the reference's signature
// (include/utils/Proto_LevelMultigridSolver.H:20-51): FAS V(6,6), lambda = 0.5/spectralRadius,
// 10 bottom sweeps, stop when res < tol*res0 (max norm). The layout must tile a periodic cube
// [0, n-1]^3 with dx = 1/n and refinement ratio 2; solve() gathers the level's valid cells, runs
// the device solver (pb_fas) and scatters the solution back. Bitwise the reference's solver.
// ---------------------------------------------------------------------------------------------
template <template <typename, MemType> class OpType, typename T = double, MemType MEM = DEVICE>
class LevelMultigridSolver {
    static_assert(std::is_same<OpType<T, MEM>, BoxOp_Laplace<double, DEVICE>>::value,
                  "the device FAS solver implements BoxOp_Laplace<double>");

public:
    LevelMultigridSolver(DisjointBoxLayout& layout, Point refRatio, int numLevels, T dx) { define(layout, refRatio, numLevels, dx); }
    void define(DisjointBoxLayout& layout, Point refRatio, int numLevels, T dx)
    {
        const Box& d = layout.domain().box;
        const int n = d.size(0);
        if (refRatio != Point::Ones(2) || d.low() != Point::Zeros() || d.size(1) != n || d.size(2) != n ||
            !layout.domain().periodic[0] || !layout.domain().periodic[1] || !layout.domain().periodic[2] || dx != 1.0 / n)
            throw Error(PB_ERR_UNSUPPORTED, "LevelMultigridSolver: periodic cube [0,n-1]^3, dx = 1/n, ratio 2 expected");
        m_layout = layout;
        pb_fas* h = nullptr;
        check(pb_fas_create(n, numLevels, &h), "LevelMultigridSolver::define");
        m_h = std::shared_ptr<pb_fas>(h, [](pb_fas* m) { pb_fas_destroy(m); });
        m_state = std::make_shared<BoxData<double, 1, DEVICE>>(d);
        m_force = std::make_shared<BoxData<double, 1, DEVICE>>(d);
    }
    // drives L(state) + force to zero from the given state; returns the last residual norm
    T solve(LevelBoxData<T>& state, LevelBoxData<T>& force, int maxIter, T tolerance)
    {
        for (size_t i = 0; i < state.size(); i++) {
            state[i].copyTo(*m_state, m_layout[i]);
            force[i].copyTo(*m_force, m_layout[i]);
        }
        std::vector<double> hist(maxIter + 1);
        int it = 0;
        check(pb_fas_solve(m_h.get(), m_force->dp(), m_state->dp(), maxIter, tolerance, &it, hist.data(), 0),
              "LevelMultigridSolver::solve");
        for (size_t i = 0; i < state.size(); i++) {
            BoxData<T> p = state[i];
            m_state->copyTo(p, m_layout[i]);
        }
        state.exchange();
        m_hist.assign(hist.begin(), hist.begin() + it + 1);
        return (T)hist[it];
    }
    const std::vector<double>& history() const { return m_hist; }

private:
    DisjointBoxLayout m_layout;
    std::shared_ptr<pb_fas> m_h;
    std::shared_ptr<BoxData<double, 1, DEVICE>> m_state, m_force;
    std::vector<double> m_hist;
};

} // namespace Proto
