// Level data: a patch layout in one device slab, its ghost exchange, and batched stencil steps.
//
// Reference counterparts (paths within the reference project):
//   LevelBoxData::define / exchange ........ include/base/implem/Proto_LevelBoxDataImplem.H:63-106, 315-329
//   LevelExchangeCopier::buildMotionPlans .. include/base/implem/Proto_LevelBoxDataImplem.H:900-951
//   Copier::makeItSoLocal .................. include/base/implem/Proto_CopierImplem.H:172-181
// The reference launches one copy kernel per motion item (up to 26 per patch) after a barrier.
// Here the motion plan is built once on the host (any disjoint tiling, uneven patch sizes
// allowed, periodic images included) and one kernel launch executes every item of the level.
#include <algorithm>
#include <cstring>
#include <vector>

#include "pb_internal.cuh"
#include "pb_stencil_impl.cuh"

namespace pb {

struct MotionItem {
    long long dOff, sOff;      // slab offsets of the destination / source patch (component 0)
    long long dvol, svol;      // grown-box volumes (component stride)
    int dlo[3], dS[3];         // destination grown box: low corner, extents
    int slo[3], sS[3];         // source grown box
    int rlo[3], rn[3];         // region, destination coordinates
    int sh[3];                 // source point = destination point - sh
};

__global__ void __launch_bounds__(256) k_exchange(double* slab, const MotionItem* __restrict__ items, int ncomp)
{
    const MotionItem it = items[blockIdx.x];
    const long long total = (long long)it.rn[0] * it.rn[1] * it.rn[2];
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        int x = it.rlo[0] + (int)(i % it.rn[0]);
        long long q = i / it.rn[0];
        int y = it.rlo[1] + (int)(q % it.rn[1]);
        int z = it.rlo[2] + (int)(q / it.rn[1]);
        long long di = (x - it.dlo[0]) + (long long)it.dS[0] * ((y - it.dlo[1]) + (long long)it.dS[1] * (z - it.dlo[2]));
        int sx = x - it.sh[0], sy = y - it.sh[1], sz = z - it.sh[2];
        long long si = (sx - it.slo[0]) + (long long)it.sS[0] * ((sy - it.slo[1]) + (long long)it.sS[1] * (sz - it.slo[2]));
        for (int c = 0; c < ncomp; c++) slab[it.dOff + c * it.dvol + di] = slab[it.sOff + c * it.svol + si];
    }
}

// One tile = a run of whole z-planes of one patch's valid box.
struct PatchTile {
    long long off;             // slab offset of the patch
    int glo[3], gS[3];         // grown box low corner and extents
    int vlo[3], vn[3];         // valid box low corner and extents
    int z0, nz;                // planes of the valid box this tile covers
};

template <class S>
__global__ void __launch_bounds__(256) k_level_star(const double* __restrict__ u, double* out,
                                                    const PatchTile* __restrict__ tiles, Coefs<double> cf, double a,
                                                    int euler)
{
    const PatchTile t = tiles[blockIdx.x];
    const long long Sx = t.gS[0], Sxy = (long long)t.gS[0] * t.gS[1];
    const long long total = (long long)t.vn[0] * t.vn[1] * t.nz;
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        int x = (int)(i % t.vn[0]);
        long long q = i / t.vn[0];
        int y = (int)(q % t.vn[1]);
        int z = t.z0 + (int)(q / t.vn[1]);
        long long gi = t.off + (x + t.vlo[0] - t.glo[0]) + Sx * (y + t.vlo[1] - t.glo[1]) + Sxy * (z + t.vlo[2] - t.glo[2]);
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < S::NT; j++) {
            const long long o = S::off(j, 0) + Sx * S::off(j, 1) + Sxy * S::off(j, 2);
            acc = dadd(acc, dmul(cf.c[j], __ldg(u + gi + o)));
        }
        double c = __ldg(u + gi);
        out[gi] = euler ? dadd(c, dmul(a, acc)) : acc;
    }
}

} // namespace pb

struct pb_level {
    std::vector<pb::Box3> patches;
    int ghost[3];
    pb::Box3 domain;
    int periodic[3];
    int ncomp;
    std::vector<long long> offsets;
    long long slab_elems;
    std::vector<pb::MotionItem> items;
    pb::MotionItem* d_items = nullptr;
    std::vector<pb::PatchTile> tiles;
    pb::PatchTile* d_tiles = nullptr;
    int device = 0;
};

using namespace pb;

static void build_items(pb_level* lv)
{
    const int np = (int)lv->patches.size();
    long long L[3];
    for (int d = 0; d < 3; d++) L[d] = bsize(lv->domain, d);
    for (int i = 0; i < np; i++) {
        const Box3& vi = lv->patches[i];
        Box3 gi;
        for (int d = 0; d < 3; d++) { gi.lo[d] = vi.lo[d] - lv->ghost[d]; gi.hi[d] = vi.hi[d] + lv->ghost[d]; }
        for (int j = 0; j < np; j++) {
            const Box3& vj = lv->patches[j];
            Box3 gj;
            for (int d = 0; d < 3; d++) { gj.lo[d] = vj.lo[d] - lv->ghost[d]; gj.hi[d] = vj.hi[d] + lv->ghost[d]; }
            for (int sz = -1; sz <= 1; sz++)
                for (int sy = -1; sy <= 1; sy++)
                    for (int sx = -1; sx <= 1; sx++) {
                        int s[3] = {sx, sy, sz};
                        bool okp = true;
                        for (int d = 0; d < 3; d++) okp &= (s[d] == 0 || lv->periodic[d]);
                        if (!okp) continue;
                        if (i == j && sx == 0 && sy == 0 && sz == 0) continue;
                        Box3 img;
                        int sh[3];
                        for (int d = 0; d < 3; d++) {
                            sh[d] = (int)(s[d] * L[d]);
                            img.lo[d] = vj.lo[d] + sh[d];
                            img.hi[d] = vj.hi[d] + sh[d];
                        }
                        Box3 r = intersect(img, gi);
                        if (bempty(r)) continue;
                        MotionItem m;
                        m.dOff = lv->offsets[i];
                        m.sOff = lv->offsets[j];
                        m.dvol = bvol(gi);
                        m.svol = bvol(gj);
                        for (int d = 0; d < 3; d++) {
                            m.dlo[d] = gi.lo[d];
                            m.dS[d] = (int)bsize(gi, d);
                            m.slo[d] = gj.lo[d];
                            m.sS[d] = (int)bsize(gj, d);
                            m.rlo[d] = r.lo[d];
                            m.rn[d] = (int)bsize(r, d);
                            m.sh[d] = sh[d];
                        }
                        lv->items.push_back(m);
                    }
        }
    }
}

static void build_tiles(pb_level* lv)
{
    const int np = (int)lv->patches.size();
    for (int i = 0; i < np; i++) {
        const Box3& v = lv->patches[i];
        PatchTile t;
        t.off = lv->offsets[i];
        for (int d = 0; d < 3; d++) {
            t.glo[d] = v.lo[d] - lv->ghost[d];
            t.gS[d] = (int)bsize(v, d) + 2 * lv->ghost[d];
            t.vlo[d] = v.lo[d];
            t.vn[d] = (int)bsize(v, d);
        }
        // about 4K points per tile
        int plane = t.vn[0] * t.vn[1];
        int nzt = std::max(1, 4096 / std::max(1, plane));
        for (int z0 = 0; z0 < t.vn[2]; z0 += nzt) {
            t.z0 = z0;
            t.nz = std::min(nzt, t.vn[2] - z0);
            lv->tiles.push_back(t);
        }
    }
}

extern "C" {

int pb_level_create(const pb_box* patches, int npatch, const int ghost[3], pb_box domain, const int periodic[3],
                    int ncomp, pb_level** out)
{
    if (!patches || npatch < 1 || !ghost || !out || ncomp < 1) return PB_ERR_ARG;
    pb_level* lv = new (std::nothrow) pb_level;
    if (!lv) return PB_ERR_NOMEM;
    lv->domain = to_box(domain);
    lv->ncomp = ncomp;
    for (int d = 0; d < 3; d++) {
        lv->ghost[d] = ghost[d];
        lv->periodic[d] = periodic ? (periodic[d] != 0) : 0;
        if (ghost[d] < 0 || (lv->periodic[d] && ghost[d] > bsize(lv->domain, d))) { delete lv; return PB_ERR_ARG; }
    }
    long long off = 0;
    for (int i = 0; i < npatch; i++) {
        Box3 b = to_box(patches[i]);
        if (bempty(b) || !contains_box(lv->domain, b)) { delete lv; return PB_ERR_BOX; }
        lv->patches.push_back(b);
        lv->offsets.push_back(off);
        long long gv = 1;
        for (int d = 0; d < 3; d++) gv *= bsize(b, d) + 2 * ghost[d];
        off += gv * ncomp;
        off = (off + 31) / 32 * 32;   // every patch starts 256-byte aligned
    }
    lv->slab_elems = off;
    build_items(lv);
    build_tiles(lv);
    cudaGetDevice(&lv->device);
    if (!lv->items.empty()) {
        if (cudaMalloc(&lv->d_items, lv->items.size() * sizeof(MotionItem)) != cudaSuccess ||
            cudaMemcpy(lv->d_items, lv->items.data(), lv->items.size() * sizeof(MotionItem), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            cudaFree(lv->d_items);
            delete lv;
            return PB_ERR_CUDA;
        }
    }
    if (cudaMalloc(&lv->d_tiles, lv->tiles.size() * sizeof(PatchTile)) != cudaSuccess ||
        cudaMemcpy(lv->d_tiles, lv->tiles.data(), lv->tiles.size() * sizeof(PatchTile), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        cudaFree(lv->d_items);
        cudaFree(lv->d_tiles);
        delete lv;
        return PB_ERR_CUDA;
    }
    *out = lv;
    return PB_OK;
}

int pb_level_destroy(pb_level* lv)
{
    if (!lv) return PB_OK;
    cudaFree(lv->d_items);
    cudaFree(lv->d_tiles);
    delete lv;
    return PB_OK;
}

int pb_level_layout(const pb_level* lv, long long* offsets, long long* slab_elems, int* nitems)
{
    if (!lv) return PB_ERR_ARG;
    if (offsets) std::memcpy(offsets, lv->offsets.data(), lv->offsets.size() * sizeof(long long));
    if (slab_elems) *slab_elems = lv->slab_elems;
    if (nitems) *nitems = (int)lv->items.size();
    return PB_OK;
}

int pb_level_exchange_f64(const pb_level* lv, double* slab, void* stream)
{
    if (!lv || !slab) return PB_ERR_ARG;
    if (lv->items.empty()) return PB_OK;
    k_exchange<<<(unsigned)lv->items.size(), 256, 0, (cudaStream_t)stream>>>(slab, lv->d_items, lv->ncomp);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

int pb_level_stencil_f64(const pb_level* lv, const pb_stencil* s, int epilogue, const double* u_slab, double* out_slab,
                         double scale, double a, void* stream)
{
    if (!lv || !s || !u_slab || !out_slab) return PB_ERR_ARG;
    if (epilogue != 0 && epilogue != PB_EPI_EULER) return PB_ERR_ARG;
    if (lv->ncomp != 1) return PB_ERR_UNSUPPORTED;
    int nterms = 0, shape = 0;
    pb_box span;
    pb_stencil_info(s, &nterms, &span, &shape);
    if (shape != 1 && shape != 2) return PB_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; d++)
        if (-span.lo[d] > lv->ghost[d] || span.hi[d] > lv->ghost[d]) return PB_ERR_GHOST;
    double c[13];
    stencil_coefs(s, c, 13);
    Coefs<double> cf;
    for (int j = 0; j < nterms; j++) cf.c[j] = (scale != 1.0) ? c[j] * scale : c[j];
    cudaStream_t st = (cudaStream_t)stream;
    unsigned nb = (unsigned)lv->tiles.size();
    if (shape == 1) k_level_star<ShapeLap7><<<nb, 256, 0, st>>>(u_slab, out_slab, lv->d_tiles, cf, a, epilogue == PB_EPI_EULER);
    else k_level_star<ShapeLap13><<<nb, 256, 0, st>>>(u_slab, out_slab, lv->d_tiles, cf, a, epilogue == PB_EPI_EULER);
    PB_LAUNCH_CHECK();
    return PB_OK;
}

} // extern "C"
