// Proto_B200_Forall.cuh — the reference's pointwise operators (forall, forall_p, forallInPlace,
// forallInPlace_p, forallOp*) over device BoxData, for callers compiled with nvcc.
//
// Reference: include/base/Proto_Forall.H:14-369 (interface), implem/Proto_ForallImplem.H (launch).
// The caller writes its pointwise function the reference's way,
//
//     PROTO_KERNEL_START
//     void consToPrim_temp(Var<double, 5>& W, const Var<double, 5>& U, double gamma) { ... }
//     PROTO_KERNEL_END(consToPrim_temp, consToPrim)
//
// or as a lambda `[=] PROTO_LAMBDA (Var<double>& u, ...) { ... }` (nvcc --extended-lambda), and
// calls forall<double, 5>(consToPrim, U, gamma) exactly as with the reference. A Var is the point's
// view of one BoxData: operator()(c) is component c at that point. Arguments are BoxData (one Var
// each) or values passed through unchanged (scalars, Point, Box). Domains follow the reference: the
// output (or, in place, the work) covers the intersection of every BoxData argument's box, or the
// Box given explicitly (intersected with the in-place arguments' boxes).
//
// The kernel is a grid-stride loop over the domain with consecutive threads on consecutive x cells
// (coalesced), 256 threads a block, at most 8 blocks per SM resident; it is launched on the legacy
// default stream like the rest of this C++ layer. One kernel per call: the reference launches one
// too (with a block per (y, z) row), so fusing several pointwise steps is the caller's choice of
// function body.
#pragma once
#include "Proto_B200.H"

#ifndef __CUDACC__
#error "Proto_B200_Forall.cuh holds device code: compile the including file with nvcc"
#endif

#define PROTO_KERNEL_START inline __host__ __device__
#define PROTO_KERNEL_END(local_name, app_name)                                               \
    struct struct_##local_name {                                                             \
        template <typename... Ts>                                                            \
        inline __host__ __device__ void operator()(Ts&&... args) const { local_name(args...); } \
        const char* myname = #app_name;                                                      \
    };                                                                                       \
    static struct_##local_name app_name;
#define PROTO_LAMBDA __host__ __device__

namespace Proto {

// The point's view of a BoxData<T, C>: component c at this point is p[c * cstride].
template <typename T, unsigned int C = 1, MemType MEM = DEVICE, unsigned int D = 1, unsigned int E = 1>
struct Var {
    T* p;
    long long cstride;
    __host__ __device__ T& operator()(unsigned int c, unsigned int d = 0, unsigned int e = 0) const
    {
        return p[(c + C * d + C * D * e) * cstride];
    }
};

namespace forall_detail {

template <typename T, unsigned int C>
struct View {   // a BoxData argument, passed to the kernel by value
    T* base;
    int lo0, lo1, lo2, sx, sy;
    long long cstride;
    __device__ Var<T, C> at(int x, int y, int z) const
    {
        return Var<T, C>{base + (x - lo0) + (long long)sx * ((y - lo1) + (long long)sy * (z - lo2)), cstride};
    }
};

template <typename A>
struct Arg {                               // a value argument: passed through
    using type = A;
    static type make(const A& a) { return a; }
    static Box box(const A&) { return Box(); }
    static constexpr bool is_data = false;
};
template <typename T, unsigned int C>
struct Arg<BoxData<T, C, DEVICE>> {        // a BoxData argument: its Var at each point
    using type = View<T, C>;
    static type make(const BoxData<T, C, DEVICE>& b)
    {
        const Box& bx = b.box();
        return type{const_cast<T*>(b.data()), bx.low()[0], bx.low()[1], bx.low()[2], bx.size(0), bx.size(1),
                    (long long)bx.size()};
    }
    static Box box(const BoxData<T, C, DEVICE>& b) { return b.box(); }
    static constexpr bool is_data = true;
};
template <typename A>
using arg_t = Arg<std::remove_cv_t<std::remove_reference_t<A>>>;

template <typename A>
__device__ __forceinline__ const A& at(const A& a, int, int, int) { return a; }
template <typename T, unsigned int C>
__device__ __forceinline__ Var<T, C> at(const View<T, C>& v, int x, int y, int z) { return v.at(x, y, z); }

// the function sees lvalues (a Var& parameter binds to them)
template <typename F, typename... V>
__device__ __forceinline__ void invoke(const F& f, V... v) { f(v...); }
template <typename F, typename... V>
__device__ __forceinline__ void invoke_p(const F& f, Point p, V... v) { f(p, v...); }

template <bool WITH_POINT, typename F, typename... A>
__global__ void __launch_bounds__(256) k_forall(const F f, int lo0, int lo1, int lo2, int nx, int ny, long long total,
                                                const A... args)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = lo0 + (int)(i % nx), y = lo1 + (int)((i / nx) % ny), z = lo2 + (int)(i / ((long long)nx * ny));
        if constexpr (WITH_POINT) invoke_p(f, Point(x, y, z), at(args, x, y, z)...);
        else invoke(f, at(args, x, y, z)...);
    }
}

inline Box intersect_all(Box acc, bool) { return acc; }
template <typename A, typename... R>
inline Box intersect_all(Box acc, bool first, const A& a, const R&... r)
{
    if constexpr (arg_t<A>::is_data) {
        acc = first ? arg_t<A>::box(a) : (acc & arg_t<A>::box(a));
        first = false;
    }
    return intersect_all(acc, first, r...);
}
// the intersection of the BoxData arguments' boxes
template <typename... A>
inline Box data_domain(const A&... a)
{
    return intersect_all(Box(), true, a...);
}
template <typename... A>
constexpr bool any_data() { return (arg_t<A>::is_data || ...); }

inline int sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

template <bool WITH_POINT, typename F, typename... A>
inline void launch(const F& f, const Box& dom, A&&... a)
{
    if (dom.empty()) return;
    const long long total = dom.size();
    const long long want = (total + 255) / 256, cap = (long long)sm_count() * 8;
    const int blocks = (int)std::max<long long>(1, std::min(want, cap));
    k_forall<WITH_POINT><<<blocks, 256>>>(f, dom.low()[0], dom.low()[1], dom.low()[2], dom.size(0), dom.size(1), total,
                                         arg_t<A>::make(a)...);
    check(cudaGetLastError() == cudaSuccess ? PB_OK : PB_ERR_CUDA, "forall");
}

} // namespace forall_detail

// ---- new output ------------------------------------------------------------------------------
// forall<T, C>(F, srcs...): BoxData<T, C> on the intersection of the BoxData arguments' boxes,
// F(Var<T, C>& out, Var/values of srcs...) at each point.
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forall(const Func& a_F, Srcs&&... a_srcs)
{
    static_assert(forall_detail::any_data<Srcs...>(), "forall: at least one BoxData argument sets the domain");
    BoxData<T, C, MEMTYPE> out(forall_detail::data_domain(a_srcs...));
    forall_detail::launch<false>(a_F, out.box(), out, a_srcs...);
    return out;
}
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forall(const Func& a_F, Box a_box, Srcs&&... a_srcs)
{
    BoxData<T, C, MEMTYPE> out(a_box);
    forall_detail::launch<false>(a_F, a_box, out, a_srcs...);
    return out;
}
// forall_p<T, C>(F, srcs...): F(Point& p, Var<T, C>& out, ...)
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forall_p(const Func& a_F, Srcs&&... a_srcs)
{
    static_assert(forall_detail::any_data<Srcs...>(), "forall_p: at least one BoxData argument sets the domain");
    BoxData<T, C, MEMTYPE> out(forall_detail::data_domain(a_srcs...));
    forall_detail::launch<true>(a_F, out.box(), out, a_srcs...);
    return out;
}
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forall_p(const Func& a_F, Box a_box, Srcs&&... a_srcs)
{
    BoxData<T, C, MEMTYPE> out(a_box);
    forall_detail::launch<true>(a_F, a_box, out, a_srcs...);
    return out;
}
// forallOp*: the same, with the reference's flop count and timer name (timers are off here)
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forallOp(unsigned long long, const char*, const Func& a_F, Srcs&&... a_srcs)
{
    return forall<T, C, MEMTYPE, D, E>(a_F, std::forward<Srcs>(a_srcs)...);
}
template <typename T, unsigned int C = 1, MemType MEMTYPE = DEVICE, unsigned int D = 1, unsigned int E = 1,
          typename Func, typename... Srcs>
inline BoxData<T, C, MEMTYPE> forallOp_p(unsigned long long, const char*, const Func& a_F, Srcs&&... a_srcs)
{
    return forall_p<T, C, MEMTYPE, D, E>(a_F, std::forward<Srcs>(a_srcs)...);
}

// ---- in place --------------------------------------------------------------------------------
// forallInPlace(F, srcs...): F over the intersection of the BoxData arguments' boxes; with a Box
// first, over that Box intersected with them.
template <typename Func, typename... Srcs>
inline void forallInPlace(const Func& a_F, Srcs&&... a_srcs)
{
    static_assert(forall_detail::any_data<Srcs...>(), "forallInPlace: at least one BoxData argument");
    forall_detail::launch<false>(a_F, forall_detail::data_domain(a_srcs...), a_srcs...);
}
template <typename Func, typename... Srcs>
inline void forallInPlace(const Func& a_F, Box a_box, Srcs&&... a_srcs)
{
    forall_detail::launch<false>(a_F, a_box & forall_detail::data_domain(a_srcs...), a_srcs...);
}
template <typename Func, typename... Srcs>
inline void forallInPlace_p(const Func& a_F, Srcs&&... a_srcs)
{
    static_assert(forall_detail::any_data<Srcs...>(), "forallInPlace_p: at least one BoxData argument");
    forall_detail::launch<true>(a_F, forall_detail::data_domain(a_srcs...), a_srcs...);
}
template <typename Func, typename... Srcs>
inline void forallInPlace_p(const Func& a_F, Box a_box, Srcs&&... a_srcs)
{
    forall_detail::launch<true>(a_F, a_box & forall_detail::data_domain(a_srcs...), a_srcs...);
}
template <typename Func, typename... Srcs>
inline void forallInPlaceOp(unsigned long long, const char*, const Func& a_F, Srcs&&... a_srcs)
{
    forallInPlace(a_F, std::forward<Srcs>(a_srcs)...);
}
template <typename Func, typename... Srcs>
inline void forallInPlaceOp_p(unsigned long long, const char*, const Func& a_F, Srcs&&... a_srcs)
{
    forallInPlace_p(a_F, std::forward<Srcs>(a_srcs)...);
}

} // namespace Proto
