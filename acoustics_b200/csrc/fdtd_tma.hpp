// fdtd_tma.hpp — plain data of the TMA-staged PML-shell kernel
// (fdtd_shell_tma.cuh), shared by the host code that builds its tiles and
// tensor maps (fdtd_tma.cpp) and the device code.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace fdtd {

constexpr int TMA_THREADS = 128;                    // consumer threads (4 warps) of a CTA
constexpr int TMA_BLOCK = TMA_THREADS + 32;         // + one producer warp
constexpr int TMA_STAGES = 5;
constexpr int TMA_MAX_SHAPES = 8;
// bit the shell kernel sets in the solve's dev_error flags when a stage never arrives
constexpr int FDTD_DEV_ERR_TMA_TIMEOUT = 2;

// Axis set of a tile: the axes along which every cell of the tile absorbs.
enum : int { TC_X = 1, TC_Y = 2, TC_Z = 4 };
// Buffers of a ring stage.
enum : int { TB_P = 0, TB_VX = 1, TB_VY = 2, TB_VZ = 3, TB_A0 = 4, TB_A1 = 5, TB_A2 = 6, TB_N = 7 };

// One tile of the shell: cells x in [x0, x0+nx), y in [y0, y0+ny),
// z in [zlo, zhi) of the window [z0, z0 + tz) of its shape, all with the same
// absorbing axes.
struct alignas(16) TmaTile {
    int cls;        // TC_* bits (never 0)
    int shape;      // index into TmaLaunch::shape
    int x0, nx;
    int y0, ny;
    int z0;         // multiple of 4
    int zlo, zhi;
    int pad[3];
};

// Window shape (tz x ty cells; tz / 4 * ty <= TMA_THREADS) and the byte
// offsets / sizes of the buffers of a stage (size 0: not used by the shape's tiles).
struct TmaShape {
    int tz, ty;
    int off[TB_N];
    int bytes[TB_N];
};

struct TmaLaunch {
    TmaShape shape[TMA_MAX_SHAPES];
    int nshape;
    int stage_bytes;  // bytes of one ring stage (multiple of 128)
    int ntiles;
    int pad;
};

// Everything a step needs to launch the kernel: the launch description (host
// memory), the device tile table (ordered by CTA: CTA b takes tiles
// cta_first[b] .. cta_first[b+1]-1), and the device tensor maps
// [parity of p^n][shape][TB_*] (64-byte aligned, written before any launch).
struct TmaStep {
    TmaLaunch launch;
    int grid;          // persistent CTAs
    TmaTile* d_tiles;
    int* d_cta_first;  // grid + 1 offsets
    CUtensorMap* d_maps;
};

// dynamic shared memory of the kernel: the ring, then a full and an empty mbarrier per stage
inline int tma_smem_bytes(const TmaLaunch& L) { return TMA_STAGES * L.stage_bytes + 16 * TMA_STAGES; }
// CTAs of the kernel that fit on one SM with this dynamic shared memory (fdtd_fp32.cu)
int tma_blocks_per_sm(int smem_bytes);

}  // namespace fdtd
