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

bool any_pml(const std::vector<uint8_t>& cell, int a, int b) {
    for (int i = std::max(a, 0); i < std::min(b, (int)cell.size()); ++i)
        if (cell[i]) return true;
    return false;
}

}  // namespace

bool tma_encoder_available() { return encode_tiled() != nullptr; }

void free_shell_tma(fdtd_solver* s) {
    if (!s->tma) return;
    if (s->tma->d_tiles) cudaFree(s->tma->d_tiles);
    delete s->tma;
    s->tma = nullptr;
    s->region.tma = nullptr;
}

// Tiles and maps of this solve's shell (the five-box shell of the reduced
// state: x slabs over the whole (y, z) face, y slabs over the inner x range,
// z slabs over the inner x and y ranges).  FDTD_ERR_UNSUPPORTED when the
// layout does not fit the kernel (the caller then keeps the cp.async kernel).
fdtd_status build_shell_tma(fdtd_solver* s) {
    free_shell_tma(s);
    if (!tma_encoder_available()) return (set_error(s, "cuTensorMapEncodeTiled unavailable"), FDTD_ERR_UNSUPPORTED);
    const int* N = s->N;
    const int* lo = s->interior.lo;
    const int* hi = s->interior.hi;
    for (int d = 0; d < 3; ++d)
        if (!(lo[d] > 0 && hi[d] < N[d] && lo[d] < hi[d]))
            return (set_error(s, "shell layout outside the TMA kernel's"), FDTD_ERR_UNSUPPORTED);
    constexpr int TZ0 = 64, TY0 = 8;
    // z-slab windows: [0, lo2) and [hi2 rounded down to 4, N2)
    const int zh0 = hi[2] / 4 * 4;
    const int zw = std::max((lo[2] + 3) / 4 * 4, (N[2] - zh0 + 3) / 4 * 4);
    int TZ1 = 4;
    while (TZ1 < zw) TZ1 *= 2;
    if (TZ1 > 64) return (set_error(s, "z slabs wider than the TMA kernel's windows"), FDTD_ERR_UNSUPPORTED);
    const int TY1 = 512 / TZ1;

    // x planes per tile: 16, or fewer until the tiles fill three CTAs per SM
    std::vector<TmaTile> tiles;
    for (int XS = 16; XS >= 4; XS /= 2) {
        tiles.clear();
        auto add = [&](int kind, int x0, int x1, int y0, int ny, int z0, int zlo, int zhi, int flags) {
            for (int xa = x0; xa < x1; xa += XS) {
                TmaTile t{};
                t.kind = kind;
                t.x0 = xa;
                t.nx = std::min(XS, x1 - xa);
                t.y0 = y0;
                t.ny = ny;
                t.z0 = z0;
                t.zlo = zlo;
                t.zhi = zhi;
                t.flags = flags;
                tiles.push_back(t);
            }
        };
        const auto& py = s->tab[1].pml_cell;
        const auto& pz = s->tab[2].pml_cell;
        // x slabs: every row absorbs along x; rows of the y PML also along y, z-PML cells along z
        for (int side = 0; side < 2; ++side) {
            const int xa = side ? hi[0] : 0, xb = side ? N[0] : lo[0];
            for (int y0 = 0; y0 < N[1]; y0 += TY0)
                for (int z0 = 0; z0 < N[2]; z0 += TZ0) {
                    const int ny = std::min(TY0, N[1] - y0);
                    const bool vy = any_pml(py, y0, y0 + ny), vz = any_pml(pz, z0, z0 + TZ0);
                    add(0, xa, xb, y0, ny, z0, 0, N[2], (vy ? TT_VY : 0) | (vz ? TT_VZ : 0) | (vy || vz ? TT_A2 : 0));
                }
        }
        // y slabs
        for (int side = 0; side < 2; ++side) {
            const int ya = side ? hi[1] : 0, yb = side ? N[1] : lo[1];
            for (int y0 = ya; y0 < yb; y0 += TY0)
                for (int z0 = 0; z0 < N[2]; z0 += TZ0) {
                    const bool vz = any_pml(pz, z0, z0 + TZ0);
                    add(1, lo[0], hi[0], y0, std::min(TY0, yb - y0), z0, 0, N[2], TT_VY | (vz ? TT_VZ | TT_A2 : 0));
                }
        }
        // z slabs
        for (int side = 0; side < 2; ++side) {
            const int z0 = side ? zh0 : 0, zlo = side ? hi[2] : 0, zhi = side ? N[2] : lo[2];
            for (int y0 = lo[1]; y0 < hi[1]; y0 += TY1)
                add(2, lo[0], hi[0], y0, std::min(TY1, hi[1] - y0), z0, zlo, zhi, TT_VZ | TT_A2);
        }
        if ((int)tiles.size() >= 3 * 148) break;
    }
    std::unique_ptr<TmaStep> T(new TmaStep());
    std::memset(T.get(), 0, sizeof(TmaStep));
    const unsigned all = (1u << TB_N) - 1u;
    const unsigned zs = (1u << TB_P) | (1u << TB_VZ) | (1u << TB_A0) | (1u << TB_A2);
    T->launch.shape[0] = make_shape(TZ0, TY0, all);
    T->launch.shape[1] = make_shape(TZ1, TY1, zs);
    T->launch.stage_bytes = std::max(shape_bytes(T->launch.shape[0]), shape_bytes(T->launch.shape[1]));
    T->launch.ntiles = (int)tiles.size();
    const SolveParams& P = s->hP;
    for (int c = 0; c < 2; ++c)
        for (int sh = 0; sh < 2; ++sh) {
            const TmaShape& S = T->launch.shape[sh];
            CUtensorMap* m = T->maps[c].m[sh];
            bool ok = encode(&m[TB_P], P.p[c], s, S.tz + 8, S.ty + 2) &&
                      encode(&m[TB_VZ], P.v[c][2], s, S.tz + 4, S.ty) && encode(&m[TB_A0], P.pd[0], s, S.tz, S.ty) &&
                      encode(&m[TB_A2], P.pd[2], s, S.tz, S.ty);
            if (ok && sh == 0)
                ok = encode(&m[TB_VX], P.v[c][0], s, S.tz, S.ty) && encode(&m[TB_VY], P.v[c][1], s, S.tz, S.ty + 1) &&
                     encode(&m[TB_A1], P.pd[1], s, S.tz, S.ty);
            if (!ok) return (set_error(s, "cuTensorMapEncodeTiled rejected a shell map"), FDTD_ERR_UNSUPPORTED);
        }
    const size_t tb = tiles.size() * sizeof(TmaTile);
    cudaError_t e = cudaMalloc((void**)&T->d_tiles, tb);
    if (e != cudaSuccess) {
        T->d_tiles = nullptr;
        cuda_fail(s, e, "cudaMalloc (shell tiles)");
        return e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA;
    }
    e = counted_copy(s, T->d_tiles, tiles.data(), tb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(T->d_tiles);
        cuda_fail(s, e, "copy of the shell tiles");
        return FDTD_ERR_CUDA;
    }
    s->tma = T.release();
    s->region.tma = s->tma;
    return FDTD_OK;
}

}  // namespace fdtd
