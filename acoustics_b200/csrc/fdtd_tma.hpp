// fdtd_tma.hpp — plain data of the TMA-staged PML-shell kernel
// (fdtd_shell_tma.cuh), shared by the host code that builds its tiles and
// tensor maps (fdtd_tma.cpp) and the device code.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace fdtd {

constexpr int TMA_THREADS = 128;
constexpr int TMA_STAGES = 4;
// bit the shell kernel sets in the solve's dev_error flags when a stage never arrives
constexpr int FDTD_DEV_ERR_TMA_TIMEOUT = 2;

enum : int { TT_VY = 1, TT_VZ = 2, TT_A2 = 4 };
enum : int { TB_P = 0, TB_VX = 1, TB_VY = 2, TB_VZ = 3, TB_A0 = 4, TB_A1 = 5, TB_A2 = 6, TB_N = 7 };

// One tile of the shell.
struct alignas(16) TmaTile {
    int kind;       // 0 x slab, 1 y slab, 2 z slab
    int x0, nx;     // planes [x0, x0 + nx)
    int y0, ny;     // rows [y0, y0 + ny), ny <= TY of the shape
    int z0;         // first z of the window (multiple of 4)
    int zlo, zhi;   // cells of the box in the window: z in [zlo, zhi)
    int flags;      // TT_*: y faces / z faces / third split array are read
    int pad[3];
};

// Window shape and stage layout (byte offsets of the buffers in a stage).
struct TmaShape {
    int tz, ty;
    int off[TB_N];
    int bytes[TB_N];
};

// Tensor maps of the arrays, per window shape; P and the faces depend on the
// buffer parity of the step, so the host passes the maps of this step.
struct TmaMaps {
    CUtensorMap m[2][TB_N];  // [shape][TB_*]; A0..A2 are the three split arrays
};

struct TmaLaunch {
    TmaShape shape[2];
    int stage_bytes;  // bytes of one ring stage (multiple of 128)
    int ntiles;
};

// Everything a step needs to launch the kernel (host memory of the solver):
// the maps of both buffer parities and the device tile table.
struct TmaStep {
    TmaMaps maps[2];  // [parity of p^n]
    TmaLaunch launch;
    TmaTile* d_tiles;
};

// dynamic shared memory of the kernel: the ring and one mbarrier per stage
inline int tma_smem_bytes(const TmaLaunch& L) { return TMA_STAGES * L.stage_bytes + 8 * TMA_STAGES; }

}  // namespace fdtd
