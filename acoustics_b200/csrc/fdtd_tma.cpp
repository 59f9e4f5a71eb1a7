// fdtd_tma.cpp — tiles and tensor maps of the TMA-staged PML-shell kernel
// (fdtd_shell_tma.cuh) for FP32 solves on the reduced PML state.
//
// The tensor maps are encoded with the driver's cuTensorMapEncodeTiled, reached
// through the runtime's driver entry point (the library links the CUDA runtime
// statically and does not link the driver library).  Every map describes one
// padded grid array of this solve (this GPU's memory): dimensions
// {SY, Ny + 1, Nx + 1} elements, strides {SY, SX} elements, FP32, no swizzle,
// out-of-range elements read as zero.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "fdtd_internal.hpp"
#include "fdtd_tma.hpp"

namespace fdtd {
namespace {

void cuda_fail(fdtd_solver* s, cudaError_t e, const char* what) {
    set_error(s, std::string("CUDA: ") + cudaGetErrorString(e) + " at " + what);
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
    static EncodeTiled fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiled>(f);
    }();
    return fn;
}

bool encode(CUtensorMap* m, const void* base, const fdtd_solver* s, int box_z, int box_y) {
    const cuuint64_t dims[3] = {(cuuint64_t)s->SY, (cuuint64_t)(s->N[1] + 1), (cuuint64_t)(s->N[0] + 1)};
    const cuuint64_t strides[2] = {(cuuint64_t)s->SY * 4, (cuuint64_t)s->SX * 4};
    const cuuint32_t box[3] = {(cuuint32_t)box_z, (cuuint32_t)box_y, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    return encode_tiled()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, elem,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int round128(int b) { return (b + 127) / 128 * 128; }

// Stage layout of a window shape: the buffers `used` (TB_* bits) one after the
// other, each on a 128-byte boundary.
TmaShape make_shape(int tz, int ty, unsigned used) {
    TmaShape S{};
    S.tz = tz;
    S.ty = ty;
    int bytes[TB_N] = {(ty + 2) * (tz + 8) * 4, ty * tz * 4, (ty + 1) * tz * 4, ty * (tz + 4) * 4,
                       ty * tz * 4,             ty * tz * 4, ty * tz * 4};
    int off = 0;
    for (int b = 0; b < TB_N; ++b) {
        if (!((used >> b) & 1u)) continue;
        S.off[b] = off;
        S.bytes[b] = bytes[b];
        off += round128(bytes[b]);
    }
    return S;
}
int shape_bytes(const TmaShape& S) {
    int end = 0;
    for (int b = 0; b < TB_N; ++b)
        if (S.bytes[b]) end = std::max(end, S.off[b] + round128(S.bytes[b]));
    return end;
}

}  // namespace

bool tma_encoder_available() { return encode_tiled() != nullptr; }

void free_shell_tma(fdtd_solver* s) {
    if (!s->tma) return;
    if (s->tma->d_tiles) cudaFree(s->tma->d_tiles);
    if (s->tma->d_maps) cudaFree(s->tma->d_maps);
    if (s->tma->d_cta_first) cudaFree(s->tma->d_cta_first);
    delete s->tma;
    s->tma = nullptr;
    s->region.tma = nullptr;
}

// Tiles and maps of this solve's shell, cut by absorbing axes: for every
// non-empty set of axes, the cells whose x, y and z each lie in that axis' PML
// ranges exactly for the axes of the set.  FDTD_ERR_UNSUPPORTED when the layout
// does not fit the kernel (the caller then keeps the cp.async kernel).
fdtd_status build_shell_tma(fdtd_solver* s) {
    free_shell_tma(s);
    if (!tma_encoder_available()) return (set_error(s, "cuTensorMapEncodeTiled unavailable"), FDTD_ERR_UNSUPPORTED);
    const int* N = s->N;
    const int* lo = s->interior.lo;
    const int* hi = s->interior.hi;
    for (int d = 0; d < 3; ++d)
        if (!(lo[d] > 0 && hi[d] < N[d] && lo[d] < hi[d]))
            return (set_error(s, "shell layout outside the TMA kernel's"), FDTD_ERR_UNSUPPORTED);
    struct Range {
        int a, b;
    };
    // the ranges of one axis inside / outside its PML
    auto ranges = [&](int d, bool pml) {
        std::vector<Range> r;
        if (pml) {
            r.push_back({0, lo[d]});
            r.push_back({hi[d], N[d]});
        } else {
            r.push_back({lo[d], hi[d]});
        }
        return r;
    };
    // window shape of a class: z windows start on multiples of 4
    auto shape_of = [&](bool ey, bool ez, int& tz, int& ty) -> bool {
        if (ez) {
            const int need = std::max((lo[2] + 3) / 4 * 4, (N[2] - hi[2] / 4 * 4 + 3) / 4 * 4);
            tz = 4;
            while (tz < need) tz *= 2;
            if (tz > 64) return false;
        } else {
            const int z0 = lo[2] / 4 * 4, span = hi[2] - z0;
            tz = 64;
            int waste = (span + 63) / 64 * 64 - span;
            for (int c : {32, 16}) {
                const int w = (span + c - 1) / c * c - span;
                if (w < waste) {
                    waste = w;
                    tz = c;
                }
            }
        }
        const int ty_max = 512 / tz;
        const int ey_ext = ey ? std::max(lo[1], N[1] - hi[1]) : hi[1] - lo[1];
        ty = std::min(ty_max, ey_ext);
        return ty > 0;
    };
    std::unique_ptr<TmaStep> T(new TmaStep());
    std::memset(T.get(), 0, sizeof(TmaStep));
    TmaLaunch& L = T->launch;
    int cls_shape[8];
    unsigned used[TMA_MAX_SHAPES] = {0};
    for (int cls = 1; cls < 8; ++cls) {
        const bool ex = cls & TC_X, ey = cls & TC_Y, ez = cls & TC_Z;
        int tz = 0, ty = 0;
        if (!shape_of(ey, ez, tz, ty))
            return (set_error(s, "PML slabs wider than the TMA kernel's windows"), FDTD_ERR_UNSUPPORTED);
        int sh = -1;
        for (int k = 0; k < L.nshape; ++k)
            if (L.shape[k].tz == tz && L.shape[k].ty == ty) sh = k;
        if (sh < 0) {
            sh = L.nshape++;
            L.shape[sh].tz = tz;
            L.shape[sh].ty = ty;
        }
        cls_shape[cls] = sh;
        used[sh] |= (1u << TB_P) | (1u << TB_A0);
        if (ex) used[sh] |= 1u << TB_VX;
        if (ey) used[sh] |= 1u << TB_VY;
        if (ez) used[sh] |= 1u << TB_VZ;
        if (ex || ey) used[sh] |= 1u << TB_A1;
        if (ez || (ex && ey)) used[sh] |= 1u << TB_A2;
    }
    L.stage_bytes = 0;
    for (int k = 0; k < L.nshape; ++k) {
        L.shape[k] = make_shape(L.shape[k].tz, L.shape[k].ty, used[k]);
        L.stage_bytes = std::max(L.stage_bytes, shape_bytes(L.shape[k]));
    }

    // persistent CTAs: as many as fit at once
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per_sm = std::max(1, tma_blocks_per_sm(tma_smem_bytes(L)));
    const int max_grid = sms * per_sm;
    // x planes per tile: 16, or fewer until there are three tiles per CTA to balance
    std::vector<TmaTile> tiles;
    for (int XS = 16; XS >= 4; XS /= 2) {
        tiles.clear();
        for (int cls = 1; cls < 8; ++cls) {
            const bool ex = cls & TC_X, ey = cls & TC_Y, ez = cls & TC_Z;
            const TmaShape& S = L.shape[cls_shape[cls]];
            for (const Range& rx : ranges(0, ex))
                for (const Range& ry : ranges(1, ey))
                    for (const Range& rz : ranges(2, ez)) {
                        if (rx.b <= rx.a || ry.b <= ry.a || rz.b <= rz.a) continue;
                        for (int z0 = rz.a / 4 * 4; z0 < rz.b; z0 += S.tz)
                            for (int y0 = ry.a; y0 < ry.b; y0 += S.ty)
                                for (int x0 = rx.a; x0 < rx.b; x0 += XS) {
                                    TmaTile t{};
                                    t.cls = cls;
                                    t.shape = cls_shape[cls];
                                    t.x0 = x0;
                                    t.nx = std::min(XS, rx.b - x0);
                                    t.y0 = y0;
                                    t.ny = std::min(S.ty, ry.b - y0);
                                    t.z0 = z0;
                                    t.zlo = rz.a;
                                    t.zhi = rz.b;
                                    tiles.push_back(t);
                                }
                    }
        }
        if ((int)tiles.size() >= 3 * max_grid) break;
    }
    L.ntiles = (int)tiles.size();

    // each CTA gets a list of tiles of about equal bytes (largest first, each to
    // the least loaded CTA)
    const int grid = std::max(1, std::min((int)tiles.size(), max_grid));
    std::vector<double> cost(tiles.size());
    for (size_t k = 0; k < tiles.size(); ++k) {
        const TmaShape& S = L.shape[tiles[k].shape];
        double b = 0;
        for (int q = 0; q < TB_N; ++q) b += S.bytes[q];
        cost[k] = b * (tiles[k].nx + 2);
    }
    std::vector<size_t> order(tiles.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<std::vector<size_t>> per_cta(grid);
    std::vector<std::pair<double, int>> heap;  // (load, cta), min-heap
    for (int b = 0; b < grid; ++b) heap.push_back({0.0, b});
    auto cmp = [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
        return a.first > b.first || (a.first == b.first && a.second > b.second);
    };
    std::make_heap(heap.begin(), heap.end(), cmp);
    for (size_t k : order) {
        std::pop_heap(heap.begin(), heap.end(), cmp);
        heap.back().first += cost[k];
        per_cta[heap.back().second].push_back(k);
        std::push_heap(heap.begin(), heap.end(), cmp);
    }
    std::vector<TmaTile> ordered;
    std::vector<int> first(grid + 1, 0);
    for (int b = 0; b < grid; ++b) {
        first[b] = (int)ordered.size();
        // a CTA's tiles in x order of their class: the ring runs on from one to the next
        std::sort(per_cta[b].begin(), per_cta[b].end());
        for (size_t k : per_cta[b]) ordered.push_back(tiles[k]);
    }
    first[grid] = (int)ordered.size();
    tiles.swap(ordered);
    T->grid = grid;

    // maps [parity][shape][buffer], in device memory
    std::vector<CUtensorMap> maps((size_t)2 * L.nshape * TB_N);
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    const SolveParams& P = s->hP;
    for (int c = 0; c < 2; ++c)
        for (int sh = 0; sh < L.nshape; ++sh) {
            const TmaShape& S = L.shape[sh];
            CUtensorMap* m = &maps[((size_t)c * L.nshape + sh) * TB_N];
            bool ok = encode(&m[TB_P], P.p[c], s, S.tz + 8, S.ty + 2) && encode(&m[TB_A0], P.pd[0], s, S.tz, S.ty);
            if (ok && S.bytes[TB_VX]) ok = encode(&m[TB_VX], P.v[c][0], s, S.tz, S.ty);
            if (ok && S.bytes[TB_VY]) ok = encode(&m[TB_VY], P.v[c][1], s, S.tz, S.ty + 1);
            if (ok && S.bytes[TB_VZ]) ok = encode(&m[TB_VZ], P.v[c][2], s, S.tz + 4, S.ty);
            if (ok && S.bytes[TB_A1]) ok = encode(&m[TB_A1], P.pd[1], s, S.tz, S.ty);
            if (ok && S.bytes[TB_A2]) ok = encode(&m[TB_A2], P.pd[2], s, S.tz, S.ty);
            if (!ok) return (set_error(s, "cuTensorMapEncodeTiled rejected a shell map"), FDTD_ERR_UNSUPPORTED);
        }
    const size_t tb = tiles.size() * sizeof(TmaTile), mb = maps.size() * sizeof(CUtensorMap);
    const size_t fb = first.size() * sizeof(int);
    cudaError_t e = cudaMalloc((void**)&T->d_tiles, tb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&T->d_maps, mb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&T->d_cta_first, fb);
    if (e == cudaSuccess) e = counted_copy(s, T->d_tiles, tiles.data(), tb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = counted_copy(s, T->d_maps, maps.data(), mb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = counted_copy(s, T->d_cta_first, first.data(), fb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (T->d_tiles) cudaFree(T->d_tiles);
        if (T->d_maps) cudaFree(T->d_maps);
        if (T->d_cta_first) cudaFree(T->d_cta_first);
        cuda_fail(s, e, "shell tiles and tensor maps");
        return e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA;
    }
    s->tma = T.release();
    s->region.tma = s->tma;
    return FDTD_OK;
}

}  // namespace fdtd
