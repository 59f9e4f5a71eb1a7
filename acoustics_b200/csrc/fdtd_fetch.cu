// fdtd_fetch.cu — cell read-back of PML_WaveSolver::FetchCell and
// SampleAxisAlignedSlice (PML_WaveSolver.cpp:439-458, MAC_Grid.cpp:1941-1963,
// MAC_Grid::GetCell :4182-4258): one thread per requested cell gathers its
// pressures, split pressures, face velocities, classification and stored
// Laplacian, and evaluates the ghost-face pressures of the last step with the
// same device functions the step uses.  The host turns the raw values into
// fdtd_cell records.  Compiled with -fmad=false like the step kernels, so the
// ghost-face pressures are the ones the step used, bit for bit.
#include <cmath>

#include "fdtd_coupled.cuh"
#include "fdtd_geometry.cuh"
#include "fdtd_launch.hpp"

namespace fdtd {

// cur: the parity of the next step (the solver's current one); the last step
// ran with cur ^ 1, read p^n and wrote p^{n+1} into p[cur].
template <typename T>
__global__ void __launch_bounds__(128) k_fetch_cells(const SolveParams* __restrict__ Pp, int cur,
                                                     const FetchReq* __restrict__ req, FetchVal* __restrict__ out,
                                                     int n) {
    const SolveParams& P = *Pp;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const FetchReq R = req[q];
    const long long c = R.c;
    const T* __restrict__ pc = (const T*)P.p[cur];
    // p^n of the last step: the other buffer (FP64) or p^{n+1} less the compensated increment (FP32)
    auto prev = [&](long long x) -> double {
        if constexpr (sizeof(T) == 8) return ((const double*)P.p[cur ^ 1])[x];
        else return (double)pc[x] - (double)P.dinc[x];
    };
    FetchVal o;
    o.p = (double)pc[c];
    o.p_prev = prev(c);
    for (int d = 0; d < 3; ++d) o.pdir[d] = R.a[d] ? (double)*(const T*)R.a[d] : NAN;
    for (int f = 0; f < 6; ++f) o.v[f] = R.a[3 + f] ? (double)*(const T*)R.a[3 + f] : NAN;
    o.lap = P.lapv[cur] ? (double)((const T*)P.lapv[cur])[c] : NAN;
    const uint8_t code = P.cls[c];
    const uint8_t gobj = P.gobj[c];
    o.cls = code;
    o.gobj = gobj;
    // ghost faces (MAC_Grid.cpp:4210-4227): toward -x, +x, -y, +y, -z, +z, where
    // the neighbour is bulk; RASTERIZE pressures as MAC_Grid.cpp:1188-1281 gives
    // them, FULLY_COUPLED the solved values of the last step
    int x, y, z;
    cell_ijk(P, c, x, y, z);
    const unsigned mask = (code & CLS_BULK) ? 0u : (code & CLS_MASK);
    const long long strides[3] = {P.SX, P.SY, 1};
    const int par = cur ^ 1;
    const double t = P.consts[par].t;
    for (int f = 0; f < 6; ++f) {
        o.gc[f] = -1.0;
        if (!((mask >> f) & 1u)) continue;
        const int d = f >> 1;
        const int dir = (f & 1) ? +1 : -1;
        const int nb = (d == 0 ? x : d == 1 ? y : z) + dir;
        if (nb < 0 || nb >= P.N[d]) continue;  // the classification sets no face off the grid
        const double pn = prev(c + dir * strides[d]);
        const double pos[3] = {P.cpos[0][x], P.cpos[1][y], P.cpos[2][z]};
        o.gc[f] = P.fc_rows ? fc_ghost(P, par, c, f, pn) : ghost_pressure(P, gobj, pos, d, dir, pn, t);
    }
    out[q] = o;
}

cudaError_t launch_fetch_cells(const SolveParams* dP, bool fp64, int cur, const FetchReq* req, FetchVal* out, int n,
                               cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (n + 127) / 128;
    if (fp64) k_fetch_cells<double><<<blocks, 128, 0, s>>>(dP, cur, req, out, n);
    else k_fetch_cells<float><<<blocks, 128, 0, s>>>(dP, cur, req, out, n);
    return cudaGetLastError();
}

}  // namespace fdtd
