// fdtd_device.cuh — device-side data layout and helpers shared by the FP64 and
// FP32 kernel translation units.
//
// HBM layout of one solve.  Every array (cells and the three face grids) uses
// one padded index  i*SX + j*SY + k  with z contiguous (the reference's order,
// ScalarField.cpp:86-97), SY = Nz+1 rounded up to 8 elements and
// SX = (Ny+1)*SY, over Nx+1 planes: a cell and its three low faces share an
// index, the high faces are +SX, +SY, +1, rows start on 32-byte boundaries and
// 16-byte vector accesses along z are aligned at k = 0 mod 4 (FP32) / 2 (FP64).
// Arrays are 256-byte aligned; indices returned through the C-ABI are the
// reference's dense i*Ny*Nz + j*Nz + k.
//   cls[N]      u8   bit7 bulk, bit6 valid history, bits0-5 solid-neighbour mask
//                    (bit 2d: -d side, bit 2d+1: +d side)
//   gobj[N]     u8   for ghost cells: closest object (LowestObjectDistance) | 0x80 constraint (every solid cell)
//   p[2][N]     T    pressure ping-pong (FP64: p^n and p^{n-1}, p^{n+1} overwrites p^{n-1};
//                    FP32: p^n and p^{n+1})
//   dinc[N]     f32  FP32 only: increment p^n - p^{n-1} (compensated accumulation)
//   pd[3][N]    T    PML split pressures (touched on PML cells only)
//   v[2][3][Nf] T    face velocities, double-buffered (touched on PML faces only)
// Per-axis tables replace the reference's per-cell PML coefficient lists
// (MAC_Grid.cpp:2495-2523, :2653-2677): every coefficient depends on one
// coordinate only.
#pragma once
#include "fdtd_mesh.cuh"
#include <cmath>
#include <cstdint>

#ifndef FDTD_SHELL_VZ_F32
#define FDTD_SHELL_VZ_F32 2
#endif
#ifndef FDTD_SHELL_PLANES
#define FDTD_SHELL_PLANES 8  // x planes a PML-shell thread marches over (default)
#endif
#ifndef FDTD_SHELL_RED_PLANES
#define FDTD_SHELL_RED_PLANES 8  // x planes per PML-shell thread of reduced-state solves (default)
#endif

#ifndef FDTD_MAX_OBJECTS
#define FDTD_MAX_OBJECTS 8
#endif
#ifndef FDTD_MAX_SOURCES
#define FDTD_MAX_SOURCES 4
#endif

namespace fdtd {

constexpr uint8_t CLS_BULK = 0x80;
constexpr uint8_t CLS_VALID = 0x40;
constexpr uint8_t CLS_MASK = 0x3F;
constexpr uint8_t GOBJ_CONSTRAINT = 0x80;
constexpr uint8_t GOBJ_NONE = 0x7F;

struct DevObject {
    int shape, accel_kind, motion, _pad;
    double c[3];        // current centre (a mesh's object-frame origin)
    double R[9];        // object->world rotation, row-major
    double size[3];
    double bmin[3], bmax[3], bdim[3], bcen[3];  // _bboxWorld
    double amp, t0, tau, dir[3];
    MeshView mesh;      // FDTD_SHAPE_MESH: device hierarchy and triangles
};

struct DevPlane {
    int dir, sign;
    double height;
};

struct DevSource {
    double cen[3];       // _bboxWorld.centroid
    double bmin[3], bmax[3];
    double denom;        // 2*w*w
    double t0, wt;       // offset, width in time
    double scale;        // (1/3.6836) * normalize constant
};

// Non-PML box [lo, hi) of the grid.
struct Box3 {
    int lo[3];
    int hi[3];
};

// z cells per vector group of the shell kernel for a word size (8-byte groups:
// 2 FP32 or 2 FP64 cells... FP64 uses 16 bytes)
__host__ __device__ constexpr int shell_vz(int word) { return word == 4 ? FDTD_SHELL_VZ_F32 : 2; }

// The PML shell as up to five disjoint boxes (x slabs, y slabs, the merged z-slab
// pair).  Box b covers x in [x0, x0+nx), y in [y0, y0+ny) and z in
// [za, zae) u [zb, zbe).  Along z it is cut into vector groups of vz cells
// starting at multiples of vz: gl groups cover [za, zae), the next ng - gl
// cover [zb, zbe) (groups may reach outside the ranges; those cells are
// masked).  A thread owns one group of one row for xs x planes; a CTA owns 256
// consecutive (row, group) units: tu unit tiles x tx plane tiles per box.
// block_first[] is the prefix sum of CTAs per box.
//
// The z-slab pair (box zbox) keeps its split pressures and face velocities in
// compact arrays: row (x, y) of the box at ((x - x0) * ny + (y - y0)) * zrw,
// group gi of the row at gi * vz, plus one spare group at ng * vz holding the
// high z face of the last group of each range (slot 0: first range, 1: second)
// when that face is not the next group's first slot.  Its rows are then
// contiguous instead of two short pieces per row of the grid.  Faces it
// shares with other boxes stay in the grid arrays: it reads its high x / y
// faces at the far box ends from there, and writes its low x / y faces at
// x = x0 / y = y0 to both (the x / y slabs read them as their high faces).
constexpr int SHELL_MAX_BOXES = 9;
struct ShellBoxes {
    int n, xs, vz;
    int x0[SHELL_MAX_BOXES], nx[SHELL_MAX_BOXES], y0[SHELL_MAX_BOXES], ny[SHELL_MAX_BOXES];
    int za[SHELL_MAX_BOXES], zae[SHELL_MAX_BOXES], zb[SHELL_MAX_BOXES], zbe[SHELL_MAX_BOXES];
    int gl[SHELL_MAX_BOXES], ng[SHELL_MAX_BOXES];
    int tu[SHELL_MAX_BOXES], tx[SHELL_MAX_BOXES];
    int zp[SHELL_MAX_BOXES];  // every group whole, in the box and outside the z PML
    int block_first[SHELL_MAX_BOXES + 1];
    int zbox;     // box with compact storage (-1: none)
    int zrw;      // compact row width (elements): (ng + 1) * vz
    int xy_slabs; // PML on both sides along x and y, and along z on one side at least
    long long cells;
};

struct SolveParams;
struct FcRow;
struct TmaStep;

// Precomputed order-1 MLS of one listener (static classification): the sample
// value is sum_r w_r * value_r over its rows.  A row is the pressure of a cell
// (kind 0) or the ghost pressure of one ghost face of a solid cell
// (kind 1 + 2*dim + (sign > 0)).  mode 1: the value of one cell (fewer than
// four samples); mode 2: no sample or a rank-deficient fit (0 and the error
// flag).  cells[] are the enclosing cells whose NaN test the reference's
// fit applies; a NaN there sends the listener back to the full fit.
struct LisRow {
    int cell;
    int kind;
    double w;
};
struct LisPlan {
    int mode, n, nc, cell;
    int cells[8];
};

// Per-axis PML flags of index i (one byte, read once per thread and axis by the
// shell kernel instead of four table lookups).
enum : uint8_t {
    AXF_PML = 1,        // cell i inside the PML
    AXF_FACE_LO = 2,    // face i inside the PML and not the outer face (i > 0)
    AXF_FACE_HI = 4,    // face i+1 inside the PML and not the outer face (i+1 < N)
    AXF_NEXT_PML = 8,   // cell i+1 inside the PML
    AXF_HAS_LO = 16,    // i > 0
    AXF_HAS_HI = 32     // i + 1 < N
};

// Coefficients of index i in one aligned quad: face i (velocity update and
// gradient factor) and cell i (split-pressure update and divergence factor;
// zero for i = N).  One vector load per face instead of two scalar ones.
template <typename T>
struct alignas(4 * sizeof(T)) AxisCoef {
    T vupd, vgrad, pupd, pdiv;
};

// Pointers and scalars of the hot kernels, passed by value (kernel parameters
// live in the constant bank, so the kernels issue no loads to fetch them).
template <typename T>
struct KArgs {
    int N0, N1, N2;
    unsigned sx, sy;              // padded plane and row strides (elements)
    const T* pc;                  // p^n
    T* pn;                        // p^{n+1} (FP64: also p^{n-1} in place)
    float* dinc;                  // FP32 increment
    const uint8_t* cls;
    T* pd[3];
    const T* vo[3];
    T* vn[3];
    T* zpd[3];                    // compact z-slab storage (ShellBoxes::zbox)
    const T* zvo[3];
    T* zvn[3];
    const uint8_t* axflag[3];     // AXF_* per index, [N_d + 8] (zero past N_d)
    const AxisCoef<T>* coef[3];   // [N_d + 8]
    T inv_h, c2k2, lap_scale;
    T kcalp;                      // air viscosity c alpha k
    const T* lapl;                // Laplacian of the previous step (viscosity)
    T* lapc;                      // Laplacian of this step (viscosity)
    SolveParams* P;               // device copy (for the step-constant advance)
    int cur;
    int advance;                  // the shell kernel advances consts[cur^1]
};

// Launch description of one region-split step.
struct RegionLaunch {
    Box3 interior;
    ShellBoxes shell;
    Box3 src_region;   // bounding box of the source supports inside the non-PML box
    int sources;       // launch the source kernel this step
    int ghost_cap;     // capacity of the ghost-neighbour list (0: no list kernel)
    int xb;            // x planes per interior thread
    int skip;          // kernels left out (timing of single kernels): 1 interior, 2 shell, 4 ghost list
    int red;           // FP32: the shell keeps the reduced PML state (k_pml_shell_red)
    int fc;            // FULLY_COUPLED ghost cells: solve their system before the ghost list
    const TmaStep* tma;  // reduced state: the TMA-staged shell (k_pml_shell_tma) when not null (host memory)
};

// Two copies indexed by the step parity: the kernels of a step read
// consts[cur]; one thread of the step writes consts[cur^1] for the next step.
struct StepConsts {
    double t;                       // simulation time at the start of the step
    double src_tf[FDTD_MAX_SOURCES];  // exp(-((t+k/2 - t0)/wt)^2/2)
    int64_t step;
};

// Iteration boxes of one classification (MAC_Grid::classifyCells_FAST,
// MAC_Grid.cpp:3608-3653): one per object, clipped by the constraints, and
// one per constraint; a cell outside all of them is bulk.  first[b] is the
// number of cells of the boxes before b.  The classification sweep works on
// units of 256 cells of a z row (row (i, j), chunk ch); the units a box
// reaches (a cell of the unit or a neighbour of one in the box) are rows
// u0[b][0] + [0, un[b][0]) x u0[b][1] + [0, un[b][1]), chunks u0[b][2] + [0,
// un[b][2]), and ufirst[b] counts those of the boxes before b.
constexpr int CLS_MAX_BOXES = FDTD_MAX_OBJECTS + 4;
constexpr int CLS_CHUNK = 256;
struct ClsBoxes {
    int n;
    int lo[CLS_MAX_BOXES][3];
    int rg[CLS_MAX_BOXES][3];
    long long first[CLS_MAX_BOXES + 1];
    int u0[CLS_MAX_BOXES][3];
    int un[CLS_MAX_BOXES][3];
    long long ufirst[CLS_MAX_BOXES + 1];
};

// One non-PML bulk cell one cell inside the domain edge (the Engquist-Majda
// cells, live where a side has no PML).  o[]: signed offsets of its stencil
// cells in the padded layout, by type:
//   face   (1): ii_p, ii_n, jj_p, jj_n, kk_p, kk_n, -
//   edge   (2): ii_p, jj_p, (ii_p, jj_p), ii_n, jj_n, kk_p, kk_n
//   corner (3): ii_p, jj_p, kk_p, ii_n, jj_n, kk_n, (ii_p, jj_p, kk_p)
// (ii along the first axis with a boundary normal; jj_n / jj_p and kk_n / kk_p
// clamped to the grid as the reference clamps them).  flags: bits 0-1 the
// type, bit 4+e when exterior cell e (or, e = 3, the diagonal cell) is a PML
// cell, whose next pressure comes from the PML update.
struct alignas(16) EngCell {
    unsigned c;
    int flags;
    int o[7];
    int pad;
};
constexpr int ENG_BUF = 10;   // doubles per cell: p^{n+1}, exterior values of steps n, n-1, n-2
constexpr int DEV_ERR_ENGQUIST = 4;  // an Engquist stencil met a solid cell

struct SolveParams {
    int N[3];
    int vN[3][3];         // velocity grid divisions per face orientation
    long long ncell;      // Nx*Ny*Nz
    long long SX, SY;     // padded strides of every array (elements)
    long long np;         // elements per array: (Nx+1)*SX
    long long vcount[3];
    double h, inv_h, rho, c, k;
    double c2k2;          // (c k)^2
    double lap_scale;     // 1/(h*h)
    double kcalp;         // c alpha k (air viscosity, MAC_Grid.cpp:926-930); 0 without
    int visc;             // alpha > 0: lapv holds the Laplacians of two steps
    void* lapv[2];        // T[np] each: the Laplacian of the step of that parity
    double q;             // 0.75*h  (ghost extrapolation distance, MAC_Grid.cpp:1281)
    double quarter_h;     // 0.25*h
    double bmin[3];
    int n_obj, n_plane, n_src, n_lis;
    DevObject obj[FDTD_MAX_OBJECTS];
    DevPlane plane[4];
    DevSource src[FDTD_MAX_SOURCES];
    // per-axis tables
    const uint8_t* pml_cell[3];   // [N_d]
    const uint8_t* pml_face[3];   // [N_d+1]
    const double* cpos[3];        // [N_d] cell centre coordinate
    const double* fpos[3];        // [N_d+1] face coordinate
    const double* pupd[3];        // [N_d]
    const double* pdiv[3];        // [N_d]
    const double* vupd[3];        // [N_d+1]
    const double* vgrad[3];       // [N_d+1]
    const float* pupd_f[3];
    const float* pdiv_f[3];
    const float* vupd_f[3];
    const float* vgrad_f[3];
    const uint8_t* axflag[3];     // [N_d+8] AXF_* flags (zero past N_d)
    const AxisCoef<double>* coef_d[3];  // [N_d+8]
    const AxisCoef<float>* coef_f[3];   // [N_d+8] (the same values rounded to float)
    // state
    uint8_t* cls;
    uint8_t* gobj;
    const EngCell* eng;           // [eng_n] Engquist-Majda cells (sides without PML); null when none
    double* eng_buf;              // [eng_n][ENG_BUF]
    int eng_n;
    double eng_lambda;            // c k / h
    void* p[2];
    float* dinc;
    void* pd[3];
    void* v[2][3];
    void* zpd[3];                 // compact z-slab split pressures and face velocities
    void* zv[2][3];
    long long zcount;             // elements per compact array
    StepConsts* consts;           // [2], indexed by the step parity
    int* dev_error;               // sticky device-side error flags
    const double* listeners;      // 3*n_lis
    LisRow* lis_rows;             // [n_lis][64] precomputed MLS rows (static scenes)
    LisPlan* lis_plan;            // [n_lis]
    int lis_ready;                // plans valid for the current classification
    int* solid_pml;               // solid cells inside the PML (re-zeroed every step)
    int n_solid_pml;
    double* src_ax[3];            // [n_src][N_d] per-axis spatial factors of each source:
                                  // exp(-(x_d - c_d)^2 / 2w^2) inside the source box (the
                                  // x factor times the source scale), 0 outside
    int* ghost_list;              // non-PML bulk cells with a solid neighbour
    int* ghost_count;
    int ghost_cap;
    ClsBoxes boxes;               // iteration boxes of the latest classification
    int* fresh_list;              // bulk cells without a valid history (found by the classification sweep)
    int* fresh_count;             // may exceed fresh_cap: the fresh-cell kernel then sweeps every cell
    int fresh_cap;
    int precision;                // 0 fp64, 1 fp32 compensated
    // FULLY_COUPLED ghost cells (static scenes; null under RASTERIZE)
    const FcRow* fc_rows;         // [fc_n] one row per ghost face, owners ascending, directions ascending
    const int* fc_idx;            // [np] per ghost (solid) cell: (first row << 6) | bulk-direction mask; -1 elsewhere
    double* fc_b;                 // [fc_n] right-hand side of the step
    double* fc_x;                 // [2][fc_n] ghost pressures by step parity
    double* fc_work;              // [6][fc_n] BiCGSTAB vectors
    int fc_n;
    int fc_maxit;
    int* fc_status;               // iterations of the last solve (negative: not converged)
};

// Row of the FULLY_COUPLED ghost-cell system (MAC_Grid::PML_pressureUpdateGhostCells,
// MAC_Grid.cpp:1131-1425) of one ghost face; everything but the pressures and the
// boundary acceleration is fixed for a static scene.
//   kind 0: x = pg (diagonal +1)        kind 1: constraint, x = p_neig (diagonal +1)
//   kind 2: immersed, -x + sum_u w_u x_u = -(weighted + sum_k w_k p_k + w_s r_s)
//   kind 3: immersed row whose stencil failed the condition test, -x = -pg
// with pg = p_neig - 0.75 h (g . n_cell), g = -rho a(bp, t), weighted = (g . ne) fdw,
// r_s = (g . ne) h on the boundary row of the owner.
struct FcRow {
    int owner, nbr;               // padded indices of the solid cell and its bulk neighbour
    int kind, obj, dim, sign;     // direction owner -> nbr
    int si;                       // stencil slot of the boundary (Neumann) row, -1: none
    int pad_;
    double bp[3];                 // boundary point (acceleration sample)
    double ne[3];                 // erected normal
    double fdw;                   // finite-difference weight
    double w[8];                  // interpolation weights at the image point
    int cell[8];                  // known cell of slot k (padded index), -1: none
    int unk[8];                   // unknown ghost row of slot k, -1: none
};

template <typename T>
KArgs<T> make_kargs(SolveParams* dP, const SolveParams& P, int cur);

template <>
inline KArgs<double> make_kargs<double>(SolveParams* dP, const SolveParams& P, int cur) {
    KArgs<double> A;
    A.P = dP;
    A.cur = cur;
    A.advance = 1;
    A.N0 = P.N[0]; A.N1 = P.N[1]; A.N2 = P.N[2];
    A.sx = (unsigned)P.SX;
    A.sy = (unsigned)P.SY;
    A.pc = (const double*)P.p[cur];
    A.pn = (double*)P.p[cur ^ 1];
    A.dinc = P.dinc;
    A.cls = P.cls;
    for (int d = 0; d < 3; ++d) {
        A.pd[d] = (double*)P.pd[d];
        A.vo[d] = (const double*)P.v[cur][d];
        A.vn[d] = (double*)P.v[cur ^ 1][d];
        A.zpd[d] = (double*)P.zpd[d];
        A.zvo[d] = (const double*)P.zv[cur][d];
        A.zvn[d] = (double*)P.zv[cur ^ 1][d];
        A.axflag[d] = P.axflag[d];
        A.coef[d] = P.coef_d[d];
    }
    A.inv_h = P.inv_h; A.c2k2 = P.c2k2; A.lap_scale = P.lap_scale;
    A.kcalp = P.kcalp;
    A.lapc = (double*)P.lapv[cur];
    A.lapl = (const double*)P.lapv[cur ^ 1];
    return A;
}

template <>
inline KArgs<float> make_kargs<float>(SolveParams* dP, const SolveParams& P, int cur) {
    KArgs<float> A;
    A.P = dP;
    A.cur = cur;
    A.advance = 1;
    A.N0 = P.N[0]; A.N1 = P.N[1]; A.N2 = P.N[2];
    A.sx = (unsigned)P.SX;
    A.sy = (unsigned)P.SY;
    A.pc = (const float*)P.p[cur];
    A.pn = (float*)P.p[cur ^ 1];
    A.dinc = P.dinc;
    A.cls = P.cls;
    for (int d = 0; d < 3; ++d) {
        A.pd[d] = (float*)P.pd[d];
        A.vo[d] = (const float*)P.v[cur][d];
        A.vn[d] = (float*)P.v[cur ^ 1][d];
        A.zpd[d] = (float*)P.zpd[d];
        A.zvo[d] = (const float*)P.zv[cur][d];
        A.zvn[d] = (float*)P.zv[cur ^ 1][d];
        A.axflag[d] = P.axflag[d];
        A.coef[d] = P.coef_f[d];
    }
    A.inv_h = (float)P.inv_h; A.c2k2 = (float)P.c2k2; A.lap_scale = (float)P.lap_scale;
    A.kcalp = (float)P.kcalp;
    A.lapc = (float*)P.lapv[cur];
    A.lapl = (const float*)P.lapv[cur ^ 1];
    return A;
}


// ---- batches of independent solves (fdtd_batch.cuh, fdtd_batch.cpp) ----

template <typename T>
struct BatchDesc {
    KArgs<T> a[2];       // kernel arguments by parity
    SolveParams* P;      // the member's device parameters
    Box3 interior;
    Box3 src_region;
    ShellBoxes shell;
    double* ring;        // listener rows: row (step % ring_cap) of n_lis doubles
    int ring_cap;
    int n_lis;
    int cur;             // buffer parity of the member's next step
    int active;
    int has_src;
    int ghost_cap;
    long long total;     // steps the member runs in all (the first, classifying one included)
    int halted;          // set in both tables by k_batch_advance after the member's last step
};

struct BatchTile {
    int m;       // member
    int box;     // shell box (shell tiles)
    int tz, ty, tx;
};

struct ListenerRef {
    int m, li;
};

// The interior arguments of one batch member for one step parity: the fields
// interior_tile reads, passed in the kernel's parameter bank
// (k_batch_interior_p) so that, like the single-solve kernel's, they take no
// per-thread registers.
template <typename T>
struct BatchIntMember {
    const T* pc;
    T* pn;
    float* dinc;
    const uint8_t* cls;
    unsigned sx, sy;
    T c2k2, lap_scale, kcalp;
    Box3 box;
    int tu;      // unit tiles per x-plane tile
    int member;  // descriptor index
};
constexpr int BATCH_PARAM_MEMBERS = 160;
template <typename T>
struct BatchIntParams {
    int n;                                // members listed
    int first[BATCH_PARAM_MEMBERS + 1];   // first CTA of each listed member; first[n]: all CTAs
    BatchIntMember<T> m[BATCH_PARAM_MEMBERS];
};

struct BatchLaunch {
    const void* int_params;      // host BatchIntParams<T> of this step's parity, or null (tile table)
    int int_ctas;
    void* descs;                 // BatchDesc<T>[n_members] on the device (table of this step's parity)
    void* descs_other;           // the other parity's table (k_batch_advance marks halted members in both)
    const BatchTile* int_tiles;
    int n_int;
    const BatchTile* shell_tiles;
    int n_shell;
    int n_shell_red;             // FP32: the first n_shell_red shell tiles belong to members with the reduced PML state
    const ListenerRef* refs;
    int n_refs;
    int n_members;
    int xb, xs;
    int ghost_blocks;            // per member
    int solid_blocks;            // per member (0: no member has a solid cell inside its PML)
    int src_blocks;              // per member (0: no member has a source)
};

// z-vector groups of the interior box: groups start at multiples of V = 16 /
// sizeof(T) (aligned in the padded layout); number of 32-group CTA strips
__host__ __device__ inline int interior_groups_z(const Box3& b, int V) {
    return b.hi[2] > b.lo[2] ? (b.hi[2] - 1) / V - b.lo[2] / V + 1 : 0;
}
// CTAs of 256 (row, z-group) units per x-plane tile of the interior box
__host__ __device__ inline int interior_unit_tiles(const Box3& b, int V) {
    const long long units = (long long)(b.hi[1] - b.lo[1]) * interior_groups_z(b, V);
    return b.hi[1] > b.lo[1] ? (int)((units + 255) / 256) : 0;
}

// padded index of cell (or low face) (i, j, k)
__host__ __device__ __forceinline__ long long cidx(const SolveParams& P, int i, int j, int k) {
    return i * P.SX + j * P.SY + k;
}
// (i, j, k) of a padded index
__host__ __device__ __forceinline__ void cell_ijk(const SolveParams& P, long long c, int& i, int& j, int& k) {
    i = (int)(c / P.SX);
    const long long r = c - i * P.SX;
    j = (int)(r / P.SY);
    k = (int)(r - j * P.SY);
}
// (i, j, k) of the dense (reference) index t
__host__ __device__ __forceinline__ void dense_ijk(const SolveParams& P, long long t, int& i, int& j, int& k) {
    const long long yz = (long long)P.N[1] * P.N[2];
    i = (int)(t / yz);
    const long long r = t - i * yz;
    j = (int)(r / P.N[2]);
    k = (int)(r - (long long)j * P.N[2]);
}

// Some Gaussian source contributes at the step of parity `cur` (its time
// factor has not underflowed to zero).
__device__ __forceinline__ bool sources_on(const SolveParams& P, int cur) {
    bool any = false;
    for (int s = 0; s < P.n_src; ++s) any |= P.consts[cur].src_tf[s] != 0.0;
    return any;
}

// sum_s G_s(x, t + k/2) at cell (x, y, z) (GaussianPressureSource.cpp:6-30): the
// product of the per-axis spatial factors times the step's time factor.
__device__ __forceinline__ double source_term(const SolveParams& P, int cur, int x, int y, int z) {
    double src = 0.0;
    for (int s = 0; s < P.n_src; ++s) {
        const double tf = P.consts[cur].src_tf[s];
        if (tf == 0.0) continue;
        src += ((P.src_ax[0][s * P.N[0] + x] * P.src_ax[1][s * P.N[1] + y]) * P.src_ax[2][s * P.N[2] + z]) * tf;
    }
    return src;
}

// consts[cur^1] <- the next step's constants (PML_WaveSolver.cpp:825,
// _currentTime += _timeStep; source time factors at t + k/2).
__device__ inline void advance_consts(const SolveParams& P, int cur) {
    const StepConsts& c = P.consts[cur];
    StepConsts& n = P.consts[cur ^ 1];
    const double t = c.t + P.k;
    n.t = t;
    const double ts = t + 0.5 * P.k;
    for (int s = 0; s < FDTD_MAX_SOURCES; ++s) {
        double tf = 0.0;
        if (s < P.n_src) {
            const double u = (ts - P.src[s].t0) / P.src[s].wt;
            tf = exp(-(u * u) / 2.0);
        }
        n.src_tf[s] = tf;
    }
    n.step = c.step + 1;
}

// Szudzik pairing of two cell indices (MAC_Grid.h:108-116)
__host__ __device__ inline unsigned long long szudzik(int a_, int b_) {
    const unsigned long long a = a_ < b_ ? a_ : b_;
    const unsigned long long b = a_ < b_ ? b_ : a_;
    return (a >= b ? a * a + a + b : a + b * b);
}

}  // namespace fdtd
