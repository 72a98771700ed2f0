/*
 * proto_b200.h — C ABI of the B200 (sm_100a) structured-grid library.
 *
 * Every entry point is extern "C", takes plain pointers, sizes and boxes, returns an int status
 * (PB_OK == 0, negative on error; nothing aborts or exits) and enqueues its GPU work on the
 * caller's CUDA stream (a cudaStream_t passed as void*; NULL is the legacy default stream).
 * Field pointers are DEVICE pointers owned by the caller; the library never frees them.
 *
 * Data layout is the reference's BoxData layout (include/base/Proto_BoxData.H:311 and
 * include/base/implem/Proto_BoxDataImplem.H:700-720 in the reference project): a field of C
 * components on Box [lo,hi] holds C contiguous blocks, each x fastest, linear index
 * (x-lo.x) + nx*((y-lo.y) + ny*(z-lo.z)) (Box::sindex, Proto_BoxImplem.H:76-86).
 *
 * Floating-point results of the FP64 entry points are bitwise equal to the reference's CPU path
 * (Stencil::hostApply term order, scale folded into the coefficients, one rounding per written
 * operation, no fused multiply-add).
 */
#ifndef PROTO_B200_H
#define PROTO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------------- */
enum {
    PB_OK = 0,
    PB_ERR_ARG = -1,          /* null pointer, bad count, bad enum                               */
    PB_ERR_BOX = -2,          /* box empty where forbidden, or outside the field it indexes      */
    PB_ERR_CUDA = -3,         /* a CUDA runtime call failed; pb_last_cuda_error() has the code   */
    PB_ERR_ALIGN = -4,        /* pointer alignment the call requires is not met                  */
    PB_ERR_NOMEM = -5,        /* device or host allocation failed                                */
    PB_ERR_UNSUPPORTED = -6,  /* valid request outside what this build implements                */
    PB_ERR_BUDGET = -7,       /* request exceeds the configured memory budget                    */
    PB_ERR_DEVICE = -8,       /* a kernel flagged an error (bounded wait expired, bad plan)      */
    PB_ERR_GHOST = -9         /* ghost width smaller than the stencil footprint                  */
};

typedef struct { int lo[3]; int hi[3]; } pb_box;   /* inclusive corners, like Proto::Box */

const char* pb_status_string(int status);
int pb_last_cuda_error(void);
/* Reads (and clears) the device-side error flag of the current device; synchronises the stream. */
int pb_device_check(void* stream);
/* Test hook for the failure path of every pipelined kernel (no counterpart in the reference, which
 * aborts): runs the bounded mbarrier wait those kernels use on a barrier that never completes,
 * with a limit of `tries` polls (1 .. 2^24). *expired = 1 when the wait gave up; the device error
 * flag is then set and the next pb_device_check returns PB_ERR_DEVICE. No copy is in flight and
 * the context stays usable. Synchronises the stream. */
int pb_debug_wait_expiry(unsigned int tries, int* expired, void* stream);
/* Library version string and the compute capability it was built for ("sm_100a"). */
const char* pb_version(void);

/* ---- Stencil (reference: Stencil<T>, include/base/Proto_Stencil.H:239-911) -------------------
 * A closed coefficient/offset table in insertion order (Stencil::addCoef keeps insertion order,
 * Proto_StencilImplem.H:238-276), with source ratio, destination ratio and destination shift.
 * Replaces Stencil::closeForDevice (Proto_StencilImplem.H:539-556): immutable once created. */
typedef struct pb_stencil pb_stencil;

int pb_stencil_create(const double* coefs, const int* offsets /* nterms x 3 */, int nterms,
                      const int src_ratio[3], const int dst_ratio[3], const int dst_shift[3],
                      pb_stencil** out);
int pb_stencil_destroy(pb_stencil* s);
/* Number of terms, span (bounding box of the offsets) and the specialised kernel picked
 * (0 generic table kernel, 1 seven-point Laplacian, 2 thirteen-point Laplacian). */
int pb_stencil_info(const pb_stencil* s, int* nterms, pb_box* span, int* shape);

/* Stencil::apply(src, dst, box, initToZero, scale) (Proto_StencilImplem.H:412-431, the DEVICE
 * branch protoApply at :844-895). 'box' is in the stencil's index space; an empty box (any
 * hi < lo) is inferred as indexDomain(dstBox) & indexRange(srcBox), as the reference does.
 * init_to_zero = 1 is "dst |= S(src, scale)", 0 is "dst += S(src, scale)". */
int pb_stencil_apply_f64(const pb_stencil* s, const double* src, pb_box src_box,
                         double* dst, pb_box dst_box, pb_box box, int ncomp,
                         int init_to_zero, double scale, void* stream);
int pb_stencil_apply_f32(const pb_stencil* s, const float* src, pb_box src_box,
                         float* dst, pb_box dst_box, pb_box box, int ncomp,
                         int init_to_zero, float scale, void* stream);

/* Launch-shape knobs of the star kernels (no counterpart in the reference, whose stencils run
 * on the host or as one CUDA thread per point). mode 0 picks the kernel per box (TMA z-streaming
 * above min_tma_points cells, one thread per point below), 1 forces the TMA kernel, 2 the
 * one-thread-per-point kernel; zc is the z extent per CTA (0: chosen from the occupancy so that
 * whole waves of CTAs fill the SMs); ty the CTA tile height, yb the rows and xv the adjacent x
 * points each consumer thread computes: (ty, yb, xv) one of (8,1,1), (8,2,1), (8,2,2), (4,2,2),
 * or (8,2,0), the default, which uses xv = 1 for Stencil::apply and xv = 2 for the multigrid
 * sweeps (xv = 2 applies to boxes of even x extent; others use xv = 1). min_tma_points < 0 keeps
 * the current threshold. */
int pb_star_tune_set(int mode, int zc, int ty, int yb, int xv, long long min_tma_points);
/* Depth of the TMA kernel's shared-memory ring (0: up to 2R+4 planes, 2R+3 with two x points per
 * thread, as deep as two CTAs per SM allow; else 2R+1..16) and whether
 * per-point auxiliary fields of fused kernels (multigrid right-hand sides) are staged through it
 * by TMA (1) or read from global memory (0). */
int pb_star_tune_ring(int nst, int aux_smem);

/* Fused stencil + forall (one HBM pass). With Lu = S(u, scale) on 'box' (inferred when empty):
 *   PB_EPI_AXPBY : out = a*Lu + b*u          (forall body "out = a*Lu + b*u")
 *   PB_EPI_EULER : out = u + a*Lu            (forall body "u += dt*Lu", written out of place)
 * Each result is bitwise what the reference gets from "BoxData Lu = S(u, scale)" followed by
 * forallInPlace over the same box. */
enum { PB_EPI_AXPBY = 1, PB_EPI_EULER = 2 };
int pb_stencil_apply_fused_f64(const pb_stencil* s, int epilogue, const double* u, pb_box u_box,
                               double* out, pb_box out_box, pb_box box, double scale,
                               double a, double b, void* stream);

/* ---- BoxData algebra and pointwise kernels (reference: BoxData::operatorT,
 * Proto_BoxDataImplem.H:938-985 and :1086-1110; setVal :1261-1279; copyTo :493-640) ---------- */
enum { PB_OP_ADD = 0, PB_OP_SUB = 1, PB_OP_MUL = 2, PB_OP_DIV = 3, PB_OP_ASSIGN = 4 };
/* dst op= src on dst_box & src_box, every component */
int pb_boxdata_op_f64(int op, double* dst, pb_box dst_box, const double* src, pb_box src_box,
                      int ncomp, void* stream);
/* dst op= scalar on 'region' (empty region = whole dst box) */
int pb_boxdata_scalar_f64(int op, double* dst, pb_box dst_box, pb_box region, double scalar,
                          int ncomp, void* stream);
/* copyTo(dst, srcRegion, shift): dst(p + shift) = src(p) for p in src_region & src_box with
 * p + shift in dst_box */
int pb_boxdata_copy_f64(const double* src, pb_box src_box, double* dst, pb_box dst_box,
                        pb_box src_region, const int shift[3], int ncomp, void* stream);
/* forall "out = a*x + b*y" over out_box & x_box & y_box (one component) */
int pb_forall_axpby_f64(double* out, pb_box out_box, const double* x, pb_box x_box,
                        const double* y, pb_box y_box, double a, double b, void* stream);

/* ---- Reductions (reference: Reduction<T,OP,MEM>, include/base/Proto_Reduction.H:30-185) ------
 * op: 0 Max (initial value DBL_MIN, as the reference), 1 Min, 2 Abs (absMax), 3 Sum, 4 SumAbs,
 * 5 SumSquare, over 'region' of a field on 'box' (empty region = whole box), one component.
 * pb_reduce_f64 waits for the result (Reduction::fetch); the _async form leaves the result in
 * device memory. Max/Min/Abs are exact; sums use a fixed two-level tree (deterministic run to run). */
int pb_reduce_f64(int op, const double* data, pb_box box, pb_box region, double* result, void* stream);
int pb_reduce_async_f64(int op, const double* data, pb_box box, pb_box region, double* result_dev,
                        void* stream);

/* Allocation-free reduction. No counterpart in the reference: same operations and result
 * semantics as pb_reduce_async_f64, for callers that cannot have the library call cudaMalloc
 * (stream capture in progress, device memory owned by another allocator or a fixed budget).
 * Its scratch is a static device array of 4096 partial results plus a ticket (about 33 KB per GPU
 * that loads the library, held until exit), so the region volume is limited to 4096*2048 =
 * 8,388,608 cells; larger regions return PB_ERR_BUDGET. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. Every call shares the array: calls whose kernels overlap on the GPU
 * (different streams, no ordering between them) race. The result is written to result_dev
 * (device memory); nothing is allocated and nothing synchronises. */
int pb_reduce_noalloc_f64(int op, const double* data, pb_box box, pb_box region, double* result_dev,
                          void* stream);

/* ---- Prolongation (reference: InterpStencil<T>::Constant, Proto_InterpStencilDefs.H:1-15,
 * applied by InterpStencil::apply, Proto_InterpStencilImplem.H:91-118) ----------------------
 * dst(p) (=|+=) scale*src(p/ratio) over range(src_box) & dst_box. */
int pb_interp_constant_f64(int ratio, const double* src, pb_box src_box, double* dst, pb_box dst_box,
                           int overwrite, double scale, void* stream);

/* ---- Level data and ghost exchange (reference: LevelBoxData::exchange,
 * include/base/implem/Proto_LevelBoxDataImplem.H:315-329; motion plans :900-951) ---------------
 * A level is npatch disjoint patches tiling 'domain' (uneven sizes allowed), each stored as its
 * box grown by 'ghost', all in ONE device slab: patch i starts at element offset offsets[i]
 * (pb_level_layout fills the offsets and the slab size in elements per component; components of
 * a patch are contiguous blocks). Exchange sets every ghost cell to the valid cell at its periodic
 * image, in one kernel launch for the whole level. */
typedef struct pb_level pb_level;
int pb_level_create(const pb_box* patches, int npatch, const int ghost[3], pb_box domain,
                    const int periodic[3], int ncomp, pb_level** out);
int pb_level_destroy(pb_level* lv);
int pb_level_layout(const pb_level* lv, long long* offsets /* npatch, may be NULL */,
                    long long* slab_elems, int* nitems);
int pb_level_exchange_f64(const pb_level* lv, double* slab, void* stream);
/* Halo transfer of a level sharded over several processes (reference: the remote half of
 * Copier::execute, include/base/implem/Proto_CopierImplem.H:307-460, which packs motion items into
 * MPI buffers): a plan is a list of regions, each a box of one patch of this (local) level in that
 * patch's coordinates, inside its grown box, with its element offset in a contiguous buffer
 * (components as consecutive blocks of the region's volume). Pack copies the regions' cells into the
 * buffer, unpack copies the buffer into the regions (ghost cells); one launch each. The caller moves
 * the buffers between processes (NCCL or any transport). */
typedef struct { int patch; pb_box region; long long offset; } pb_halo_item;
typedef struct pb_halo_plan pb_halo_plan;
int pb_halo_plan_create(const pb_level* lv, const pb_halo_item* items, int n, pb_halo_plan** out);
int pb_halo_plan_destroy(pb_halo_plan* plan);
/* buffer elements the plan addresses (-1 for NULL) */
long long pb_halo_plan_elems(const pb_halo_plan* plan);
int pb_halo_pack_f64(const pb_halo_plan* plan, const double* slab, double* buffer, void* stream);
int pb_halo_unpack_f64(const pb_halo_plan* plan, double* slab, const double* buffer, void* stream);
/* Batched stencil step over every patch of a level, one launch: out = u + a*S(u, scale) on each
 * patch's valid box (PB_EPI_EULER), or out = S(u, scale) (epilogue 0). u and out are slabs of the
 * same level. */
int pb_level_stencil_f64(const pb_level* lv, const pb_stencil* s, int epilogue, const double* u_slab,
                         double* out_slab, double scale, double a, void* stream);
/* 'steps' steps of exchange(u_slab), out = u + a*S(u) (PB_EPI_EULER) or S(u) (0), swap, over
 * every patch; the result ends in u_slab (tmp_slab is scratch of the same size). The launches are
 * captured into one CUDA graph on the first call and replayed while the arguments stay the same.
 * Each step's valid cells are bitwise the pair pb_level_exchange_f64 + pb_level_stencil_f64. On a
 * periodic tensor-product tiling the stencil reads face neighbours' valid cells directly (no
 * exchange pass); ghost cells of the result are then not refreshed (call pb_level_exchange_f64).
 * No counterpart in the reference, whose callers loop over exchange and per-patch stencils. */
int pb_level_steps_f64(pb_level* lv, const pb_stencil* s, int epilogue, double* u_slab, double* tmp_slab,
                       double scale, double a, int steps, void* stream);
/* Times the batched stencil per patch-size class (valid x extent) over a few tile shapes (tile
 * width along x, planes per thread) and keeps the fastest per class (blocks until done; out_slab is
 * overwritten). pb_level_tiles reports the shapes of the fused halo-2 step as (x extent, tile width
 * in cells, planes) triples. */
int pb_level_autotune_f64(pb_level* lv, const pb_stencil* s, const double* u_slab, double* out_slab,
                          double scale, void* stream);
int pb_level_tiles(const pb_level* lv, int* triples, int cap, int* n);

/* ---- Point-Jacobi multigrid (reference: LevelMultigridSolver, include/utils/implem/
 * Proto_LevelMultigridSolverImplem.H:85-433, and the archived LevelMultigrid,
 * examples/_archived/LevelMultigrid/src/LevelMultigrid.cpp) ------------------------------------
 * Periodic cell-centred N^3 grid, one box per level, levels+1 grids (N >> levels is the coarsest).
 * form PB_MG_POISSON: solves L_h phi = rhs with the reference's archived smoother written as
 *   phi += L(phi, omega/6) + (-omega*h*h/6)*rhs        (omega = 1/2 reproduces the archived solver)
 * form PB_MG_HELMHOLTZ: alpha*phi - beta*L_h phi = rhs with per-cell alpha,
 *   phi += (omega*r)/(alpha + 6*beta/h^2),  r = rhs - (alpha*phi - beta*L(phi, 1/h^2))
 * Correction-scheme V(nu1,nu2) cycles, nu_bottom sweeps on the coarsest grid, 2^3 averaging
 * restriction, piecewise-constant prolongation, max-norm residual; stops when
 * res < tol*res0 or after max_iter cycles.
 * precision PB_MG_FP64: every level in FP64, bitwise equal to the CPU reference path.
 * precision PB_MG_MIXED: FP64 residual, correction and norms around FP32 V-cycles (iterative
 * refinement); converges to the same tolerance, not bitwise. Needs nu1, nu2, levels >= 1.
 * bottom PB_MG_BOTTOM_RELAX: nu_bottom Jacobi sweeps on the coarsest grid (the reference's bottom).
 * bottom PB_MG_BOTTOM_DIRECT: exact coarsest solve through the inverse of the coarsest operator
 *   (at most 512 coarsest cells; a singular operator gets the constant (6/h^2)/N added to every
 *   entry, which fixes the solution's mean). */
enum { PB_MG_POISSON = 0, PB_MG_HELMHOLTZ = 1 };
enum { PB_MG_FP64 = 0, PB_MG_MIXED = 1 };
enum { PB_MG_BOTTOM_RELAX = 0, PB_MG_BOTTOM_DIRECT = 1 };
typedef struct {
    int n;            /* finest edge (cells); n must be divisible by 2^levels (coarsest edge >= 1) */
    int levels;       /* number of coarsenings                                                  */
    int nu1, nu2, nu_bottom;
    double omega;
    double beta;      /* Helmholtz only */
    int form;         /* PB_MG_POISSON / PB_MG_HELMHOLTZ */
    int precision;    /* PB_MG_FP64 / PB_MG_MIXED */
    int max_iter;
    double tol;
    int bottom;       /* PB_MG_BOTTOM_RELAX / PB_MG_BOTTOM_DIRECT */
} pb_mg_params;
typedef struct pb_mg pb_mg;
int pb_mg_create(const pb_mg_params* p, pb_mg** out);
int pb_mg_destroy(pb_mg* mg);
/* Device bytes held by a solver with these parameters (for admission against a budget). */
long long pb_mg_device_bytes(const pb_mg_params* p);
/* alpha: device pointer, n^3 cells (x fastest), Helmholtz form only. */
int pb_mg_set_alpha(pb_mg* mg, const double* alpha, void* stream);
/* rhs, phi: device pointers to n^3 cells (x fastest); phi holds the initial guess and receives the
 * solution. hist (host, max_iter+1 doubles, may be NULL) receives the residual norms; *iters the
 * number of V-cycles. Blocks until the solve ends. */
int pb_mg_solve(pb_mg* mg, const double* rhs, double* phi, int* iters, double* hist, void* stream);
/* pb_mg_solve with this call's cycle limit and tolerance in place of the parameters' (max_iter >= 0;
 * 0 only measures the initial residual). The archived LevelMultigrid's vCycle() and resnorm()
 * (examples/_archived/LevelMultigrid/src/LevelMultigrid.cpp:71-88,133-158) are one cycle and no
 * cycle of this. hist holds max_iter+1 doubles. Blocks. */
int pb_mg_solve_n(pb_mg* mg, const double* rhs, double* phi, int max_iter, double tol, int* iters, double* hist,
                  void* stream);
/* LevelMultigridSolver's relax on the finest level: 'sweeps' Jacobi sweeps of the solver's current
 * state (the state left by the last pb_mg_solve). Enqueued only; does not synchronise. */
int pb_mg_relax(pb_mg* mg, int sweeps, void* stream);
/* Kernel launches one V-cycle plus its residual norm issues for these parameters. */
int pb_mg_launches_per_cycle(const pb_mg_params* p);
/* Process-wide: the levels of edge <= 'edge' below the finest grid run their part of each V-cycle
 * as one single-CTA kernel instead of one launch per sweep (same arithmetic, same results);
 * 0 turns this off. Default 8 (measured faster than 16 for large solves). Applies to solvers
 * created and cycles captured afterwards. */
int pb_mg_coarse_edge(int edge);
/* Process-wide: levels of edge >= 'edge' (of the edges the two-sweep kernel is built for: 128, 192, 256,
 * 384) run each pair of consecutive Jacobi sweeps as one pass over the level (the intermediate
 * sweep stays on chip; same arithmetic, bitwise the same results); 0 turns this off. Default 128.
 * Applies to cycles captured afterwards. */
int pb_mg_relax2_min_edge(int edge);
/* Process-wide launch-shape knobs of the two-sweep pass: planes per CTA (0 = chosen from the
 * occupancy so whole waves fill the GPU), cells per thread along x (0 = the default per edge, 1 or
 * 2) and output rows per thread group (0 = the default, 2 or 4; a CTA takes two groups). For
 * tuning and tests; results do not depend on them. */
int pb_mg_relax2_shape(int zc, int cells_per_thread, int rows_per_group);

/* ---- FAS multigrid with the 4th-order flux-form Laplacian (reference: LevelMultigridSolver<
 * BoxOp_Laplace>, include/utils/implem/Proto_LevelMultigridSolverImplem.H:85-433, operator
 * examples/_common/BoxOp_Laplace.H:22-27 through BoxOp::operator(), Proto_BoxOpImplem.H:125-172) ---
 * Periodic cell-centred n^3 grid, num_levels grids (n >> (num_levels-1) the coarsest), h = 1/n.
 * Drives op(phi) + force to zero, op = -sum_d DIV_d(DiffCellToFace_d(phi)/h)/h; V(6,6) with
 * lambda = 0.5/(6/h^2) Jacobi, 10 bottom sweeps, FAS coarse force and correction; stops when
 * res < tol*res0 (max norm). Residual history and solution are bitwise the reference's. */
typedef struct pb_fas pb_fas;
/* BoxOp<T,1,0>::operator()(output, state, scale) of BoxOp_Laplace on one box (reference:
 * include/base/implem/Proto_BoxOpImplem.H:130-175 with examples/_common/BoxOp_Laplace.H:22-27):
 * out = ((0 + sum_d DIV_d(DiffCellToFace(d, Lo, 4)(state) / dx) / dx) * flux_scale) * scale (the
 * last product only when scale != 1), on 'range' (empty: all of out_box). state (on state_box) must
 * cover range grown by 2 (PB_ERR_GHOST). Bitwise the reference's operator. Enqueued only. */
int pb_boxop_laplace_f64(const double* state, pb_box state_box, double* out, pb_box out_box, pb_box range, double dx,
                         double flux_scale, double scale, void* stream);
int pb_fas_create(int n, int num_levels, pb_fas** out);
int pb_fas_destroy(pb_fas* m);
/* force, phi: device n^3 (x fastest); phi is the initial guess and receives the solution; hist
 * (host, max_iter+1, may be NULL) the residual norms; *iters the cycles run. Blocks. */
int pb_fas_solve(pb_fas* m, const double* force, double* phi, int max_iter, double tol, int* iters,
                 double* hist, void* stream);

/* ---- Serving engine (no counterpart in the reference, which solves one grid at a time) ----------
 * Periodic Poisson/Helmholtz solves of different edges, solved together: each admitted solve keeps
 * its hierarchy on the device; one pb_serve_step runs one V-cycle for every in-flight solve, each
 * cycle phase one launch for all of them, the whole step one CUDA graph. The engine's precision is
 * PB_MG_MIXED (FP32 cycle, FP64 residual, correction and norm) or PB_MG_FP64 (every level FP64,
 * the reference's arithmetic; nu1 + nu2 must be even). Solves are admitted between steps while the HBM
 * budget allows, up to max(2, max_active / 4) at a time with their right-hand side on its way to
 * the device (an upload stream of its own; hierarchies come from a stream-ordered pool of the
 * engine). An admitted solve takes a free slot in the same step when no requests are queued (light
 * load), else in the first step after its upload has landed (uploads overlap the running cycles).
 * Solves are retired when their max-norm residual drops below tol times the first one, as failed
 * after max_cycles cycles, and as failed at once when a residual is not finite (a NaN or infinite
 * right-hand side, or a diverging solve), without disturbing the other solves. Per solve
 * the arithmetic is pb_mg's solver's of the same precision (constant alpha, levels = every
 * halving, bottom = nu_bottom sweeps), so each result is the same alone and in any mix.
 * An edge must halve down to <= 16 (n = m * 2^k with m <= 16). */
enum { PB_SERVE_WAITING = 0, PB_SERVE_ACTIVE = 1, PB_SERVE_DONE = 2, PB_SERVE_FAILED = 3 };
typedef struct {
    long long hbm_budget;   /* bytes of solver hierarchies the engine may hold                     */
    int max_active;         /* solves in flight (1..256)                                           */
    int nu1, nu2, nu_bottom;
    double omega;
    double tol;             /* relative max-norm residual                                          */
    int max_cycles;         /* a solve still above tol after this many cycles is retired as failed */
    int precision;          /* PB_MG_MIXED / PB_MG_FP64                                            */
} pb_serve_params;
typedef struct {
    int n;                  /* edge                                                                */
    int form;               /* PB_MG_POISSON (L_h u = rhs) / PB_MG_HELMHOLTZ (alpha u - beta L_h u = rhs) */
    double alpha, beta;     /* Helmholtz scalars                                                   */
    const double* rhs;      /* host, n^3 (x fastest); read when the solve is admitted              */
    double* out;            /* host, n^3; receives the solution (initial guess zero)               */
} pb_serve_request;
typedef struct pb_serve pb_serve;
int pb_serve_create(const pb_serve_params* p, pb_serve** out);
int pb_serve_destroy(pb_serve* sv);
/* Queues a request; rhs and out must stay valid until its ticket completes. PB_ERR_BUDGET if one
 * solve of this edge alone exceeds the budget. */
int pb_serve_submit(pb_serve* sv, const pb_serve_request* q, long long* ticket);
/* Admits what fits, runs one cycle for every in-flight solve and retires the finished ones; a
 * retired solve's result is copied to its out buffer in the background. *active counts solves in
 * flight plus results still on their way, *waiting the queued solves plus those whose right-hand
 * side is still uploading (keep stepping while either is non-zero); active / waiting may be NULL. */
int pb_serve_step(pb_serve* sv, int* active, int* waiting);
/* Tickets completed since the last poll (up to cap): their results are in their out buffers. */
int pb_serve_poll(pb_serve* sv, long long* tickets, int cap, int* n);
/* state PB_SERVE_* (DONE / FAILED from the poll that reports the ticket on), cycles run, last
 * relative residual. */
int pb_serve_status(const pb_serve* sv, long long ticket, int* state, int* cycles, double* rel_res);
/* Host wall time spent so far per stage of pb_serve_step (seconds: admission, work-list build,
 * first residual pass of new solves, the cycle graph including its wait, retirement) and the number
 * of steps that ran a cycle. */
int pb_serve_timing(const pb_serve* sv, double* seconds5, long long* steps);
/* Bytes of hierarchies held (in use and cached for reuse). */
long long pb_serve_device_bytes(const pb_serve* sv);
/* Bytes one solve of edge n holds in a mixed-precision engine (-1 if n is not servable). */
long long pb_serve_request_bytes(int n);
/* The same for an engine of the given precision (PB_MG_MIXED / PB_MG_FP64). */
long long pb_serve_hierarchy_bytes(int n, int precision);

#ifdef __cplusplus
}
#endif
#endif /* PROTO_B200_H */
