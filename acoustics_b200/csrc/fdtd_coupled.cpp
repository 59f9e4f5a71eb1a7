// fdtd_coupled.cpp — FULLY_COUPLED ghost-cell rows
// (MAC_Grid::PML_pressureUpdateGhostCells, MAC_Grid.cpp:1131-1425, the branch
// `use_immerse_interface`).
//
// For every ghost face (a solid cell with a bulk neighbour) the reference
// reflects the face position against the closest body, interpolates the
// pressure at the image point from its 8 enclosing cells with a trilinear
// polynomial (MAC_Grid.cpp:4444-4510; a cell that is the ghost cell itself
// contributes a Neumann row at the boundary point, a cell that is another
// ghost cell contributes its ghost face nearest to the image point, whose
// pressure is an unknown of the same system) and couples all ghost faces in one
// sparse system.  The interpolation weights solve V^T w = v^T, V the 8 x 8
// Vandermonde matrix of the stencil and v the row of the image point; a
// stencil whose condition number exceeds CONDN_LIM = 25 and that contains the
// Neumann row falls back to the rasterized value.  All of this depends on the
// geometry only, so it is computed here once per classification (once for a
// static scene, every step for moving bodies); each step builds the right-hand
// side and solves the system on the device (fdtd_coupled.cuh).  Mesh bodies are
// reflected with their hierarchy in host memory.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fdtd_c.h"
#include "fdtd_geometry.cuh"
#include "fdtd_internal.hpp"

using namespace fdtd;

#define CUDA_TRY(s, expr)                                                                   \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) {                                                            \
            set_error((s), std::string("CUDA: ") + cudaGetErrorString(_e) + " at " #expr); \
            return _e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA;          \
        }                                                                                   \
    } while (0)

namespace {

constexpr double CONDN_LIM = 25.0;  // Wavesolver_ConstantsAndTypes.h:98

// FillVandermondeRegular / FillVandermondeBoundary in the scaled coordinates of
// FillVandermonde*S: (x - origin) / h + 0.5 (MAC_Grid.cpp:4444-4510).
void vdm_regular(const double pos[3], const double org[3], double h, double row[8]) {
    double q[3];
    for (int d = 0; d < 3; ++d) {
        q[d] = pos[d];
        q[d] -= org[d];
        q[d] /= h;
        q[d] += 0.5;
    }
    const double x = q[0], y = q[1], z = q[2];
    row[0] = x * y * z;
    row[1] = x * y;
    row[2] = x * z;
    row[3] = y * z;
    row[4] = x;
    row[5] = y;
    row[6] = z;
    row[7] = 1;
}

void vdm_boundary(const double pos[3], const double nrm[3], const double org[3], double h, double row[8]) {
    double q[3];
    for (int d = 0; d < 3; ++d) {
        q[d] = pos[d];
        q[d] -= org[d];
        q[d] /= h;
        q[d] += 0.5;
    }
    const double x = q[0], y = q[1], z = q[2], nx = nrm[0], ny = nrm[1], nz = nrm[2];
    row[0] = nx * y * z + ny * x * z + nz * x * y;
    row[1] = nx * y + ny * x;
    row[2] = nx * z + nz * x;
    row[3] = ny * z + nz * y;
    row[4] = nx;
    row[5] = ny;
    row[6] = nz;
    row[7] = 0;
}

// One-sided Jacobi SVD of the 8 x 8 matrix A (row-major, overwritten by U Sigma):
// A = U diag(sig) W^T.  Returns sig (unsorted) and W (row-major).
void jacobi_svd8(double A[64], double sig[8], double W[64]) {
    for (int i = 0; i < 64; ++i) W[i] = (i % 9 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 7; ++p)
            for (int q = p + 1; q < 8; ++q) {
                double a = 0.0, b = 0.0, g = 0.0;
                for (int i = 0; i < 8; ++i) {
                    a += A[i * 8 + p] * A[i * 8 + p];
                    b += A[i * 8 + q] * A[i * 8 + q];
                    g += A[i * 8 + p] * A[i * 8 + q];
                }
                if (g == 0.0 || std::fabs(g) <= 1e-300) continue;
                off = std::max(off, std::fabs(g) / std::sqrt(a * b));
                const double zeta = (b - a) / (2.0 * g);
                const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < 8; ++i) {
                    const double x = A[i * 8 + p], y = A[i * 8 + q];
                    A[i * 8 + p] = c * x - s * y;
                    A[i * 8 + q] = s * x + c * y;
                    const double u = W[i * 8 + p], v = W[i * 8 + q];
                    W[i * 8 + p] = c * u - s * v;
                    W[i * 8 + q] = s * u + c * v;
                }
            }
        if (off < 1e-15) break;
    }
    for (int j = 0; j < 8; ++j) {
        double n = 0.0;
        for (int i = 0; i < 8; ++i) n += A[i * 8 + j] * A[i * 8 + j];
        sig[j] = std::sqrt(n);
    }
}

// w = pinv(M) v with M = V^T (the transposed stencil matrix) through its SVD;
// singular values below 8 eps sigma_max count as zero, as the default
// threshold of the reference's SVD solve.  Returns the condition number
// sigma_max / sigma_min.
double solve_weights(const double V[64], const double v[8], double w[8]) {
    double A[64], W[64], sig[8];
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) A[i * 8 + j] = V[j * 8 + i];  // M = V^T
    jacobi_svd8(A, sig, W);
    double smax = 0.0, smin = 1e300;
    for (int j = 0; j < 8; ++j) {
        smax = std::max(smax, sig[j]);
        smin = std::min(smin, sig[j]);
    }
    const double thr = 8.0 * 2.220446049250313e-16 * smax;
    // M = U S W^T with U S = A (columns); pinv(M) v = W S^-1 U^T v = W S^-2 (U S)^T v
    double c[8];
    for (int j = 0; j < 8; ++j) {
        double d = 0.0;
        for (int i = 0; i < 8; ++i) d += A[i * 8 + j] * v[i];
        c[j] = sig[j] > thr ? d / (sig[j] * sig[j]) : 0.0;
    }
    for (int i = 0; i < 8; ++i) {
        double d = 0.0;
        for (int j = 0; j < 8; ++j) d += W[i * 8 + j] * c[j];
        w[i] = d;
    }
    return smin > 0.0 ? smax / smin : INFINITY;
}

unsigned long long szudzik(long long a_, long long b_) {
    const unsigned long long a = (unsigned long long)std::min(a_, b_), b = (unsigned long long)std::max(a_, b_);
    return a >= b ? a * a + a + b : a + b * b;
}

}  // namespace

namespace fdtd {

void free_fully_coupled(fdtd_solver* s) {
    for (void* p : s->fc_alloc)
        if (p) cudaFree(p);
    s->fc_alloc.clear();
    SolveParams& P = s->hP;
    P.fc_rows = nullptr;
    P.fc_idx = nullptr;
    P.fc_b = P.fc_x = P.fc_work = nullptr;
    P.fc_status = nullptr;
    P.fc_n = 0;
}

// Rows of the FULLY_COUPLED system after a classification.
fdtd_status build_fully_coupled(fdtd_solver* s) {
    free_fully_coupled(s);
    SolveParams& P = s->hP;
    const long long np = s->np;
    std::vector<uint8_t> cls(np), gobj(np);
    CUDA_TRY(s, cudaMemcpyAsync(cls.data(), P.cls, np, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(gobj.data(), P.gobj, np, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    const int* N = s->N;
    const long long strides[3] = {s->SX, s->SY, 1};
    auto bulk = [&](long long c) { return (cls[c] & CLS_BULK) != 0; };
    auto ijk = [&](long long c, int& i, int& j, int& k) {
        i = (int)(c / s->SX);
        j = (int)((c - i * s->SX) / s->SY);
        k = (int)(c - i * s->SX - j * s->SY);
    };
    auto dense = [&](long long c) {
        int i, j, k;
        ijk(c, i, j, k);
        return ((long long)i * N[1] + j) * N[2] + k;
    };
    auto centre = [&](long long c, double x[3]) {
        int id[3];
        ijk(c, id[0], id[1], id[2]);
        for (int d = 0; d < 3; ++d) x[d] = s->tab[d].cpos[id[d]];
    };
    // ghost faces: owners ascending, directions f = 2 dim + (sign > 0) ascending
    std::vector<int> idx(np, -1);
    std::vector<FcRow> rows;
    for (int i = 0; i < N[0]; ++i)
        for (int j = 0; j < N[1]; ++j)
            for (int k = 0; k < N[2]; ++k) {
                const long long c = i * s->SX + j * s->SY + k;
                if (bulk(c)) continue;
                const int id[3] = {i, j, k};
                int mask = 0;
                for (int f = 0; f < 6; ++f) {
                    const int d = f >> 1, sg = (f & 1) ? 1 : -1;
                    const int q = id[d] + sg;
                    if (q < 0 || q >= N[d]) continue;
                    if (bulk(c + sg * strides[d])) mask |= 1 << f;
                }
                if (!mask) continue;
                idx[c] = ((int)rows.size() << 6) | mask;
                for (int f = 0; f < 6; ++f) {
                    if (!((mask >> f) & 1)) continue;
                    FcRow r;
                    std::memset(&r, 0, sizeof(r));
                    r.owner = (int)c;
                    r.dim = f >> 1;
                    r.sign = (f & 1) ? 1 : -1;
                    r.nbr = (int)(c + r.sign * strides[r.dim]);
                    r.si = -1;
                    for (int q = 0; q < 8; ++q) r.cell[q] = r.unk[q] = -1;
                    if (gobj[c] & GOBJ_CONSTRAINT) r.kind = 1;
                    else if ((gobj[c] & 0x7F) >= (unsigned)P.n_obj) r.kind = 1;  // no object: the neighbour's value
                    else r.obj = gobj[c] & 0x7F;
                    rows.push_back(r);
                }
            }
    const double h = s->h;
    const long long nrow = (long long)rows.size();
    // the ghost face of cell g nearest to a point (first in ascending key order)
    auto nearest_face = [&](long long g, const double x[3]) -> int {
        const int e = idx[g];
        if (e < 0) return -1;
        double cg[3];
        centre(g, cg);
        int best = -1;
        unsigned long long best_key = 0;
        double best_d2 = 0.0;
        for (int f = 0; f < 6; ++f) {
            if (!((e >> f) & 1)) continue;
            const int d = f >> 1, sg = (f & 1) ? 1 : -1;
            double fp[3] = {cg[0], cg[1], cg[2]};
            fp[d] += (sg > 0 ? 1.0 : -1.0) * 0.25 * h;
            double d2 = 0.0;
            for (int a = 0; a < 3; ++a) d2 += (fp[a] - x[a]) * (fp[a] - x[a]);
            const int row = (e >> 6) + __builtin_popcount((unsigned)(e & 63) & ((1u << f) - 1u));
            const unsigned long long key = szudzik(dense(g), dense(g + sg * strides[d]));
            if (best < 0 || d2 < best_d2 || (d2 == best_d2 && key < best_key)) {
                best = row;
                best_d2 = d2;
                best_key = key;
            }
        }
        return best;
    };
    // the bodies as the host queries them: mesh hierarchies in host memory
    std::vector<DevObject> hobj(P.obj, P.obj + std::max(0, P.n_obj));
    for (size_t i = 0; i < hobj.size() && i < s->objs.size(); ++i)
        if (hobj[i].shape == FDTD_SHAPE_MESH) {
            const MeshHost& M = s->meshes[s->objs[i].d.mesh];
            hobj[i].mesh = MeshView{M.nodes.data(), M.tris.data(), (int)M.nodes.size(), (int)M.tris.size()};
        }
    for (long long ri = 0; ri < nrow; ++ri) {
        FcRow& r = rows[ri];
        if (r.kind == 1) continue;
        const DevObject& o = hobj[r.obj];
        double pos[3];
        centre(r.owner, pos);
        pos[r.dim] += (r.sign > 0 ? 1.0 : -1.0) * 0.25 * h;
        double image[3], dist = 0.0;
        reflect_against_boundary(o, pos, image, r.bp, r.ne, dist);
        r.fdw = distance_to_mesh(o, pos) < 0.0 ? -2.0 * std::fabs(dist) : -std::fabs(dist);
        int nb[8];
        const int n = enclosing_neighbours(P, image, nb);
        if (n != 8) {
            r.kind = 0;
            continue;
        }
        double org[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 8; ++q) {
            double cp[3];
            centre(nb[q], cp);
            for (int d = 0; d < 3; ++d) org[d] += cp[d];
        }
        for (int d = 0; d < 3; ++d) org[d] /= 8.0;
        double V[64], v[8];
        vdm_regular(image, org, h, v);
        for (int q = 0; q < 8; ++q) {
            const long long nq = nb[q];
            if (nq == r.owner) {
                vdm_boundary(r.bp, r.ne, org, h, V + q * 8);
                r.si = q;
            } else if (idx[nq] < 0) {  // not a ghost cell: a known pressure
                double cp[3];
                centre(nq, cp);
                vdm_regular(cp, org, h, V + q * 8);
                r.cell[q] = (int)nq;
            } else {
                const int u = nearest_face(nq, image);
                const FcRow& ru = rows[u];
                double fp[3];
                centre(ru.owner, fp);
                fp[ru.dim] += (ru.sign > 0 ? 1.0 : -1.0) * 0.25 * h;
                vdm_regular(fp, org, h, V + q * 8);
                r.unk[q] = u;
            }
        }
        const double cond = solve_weights(V, v, r.w);
        if (cond > CONDN_LIM && r.si != -1) {
            r.kind = 3;
            r.si = -1;
            for (int q = 0; q < 8; ++q) {
                r.w[q] = 0.0;
                r.cell[q] = r.unk[q] = -1;
            }
        } else {
            r.kind = 2;
        }
    }
    if (nrow == 0) return FDTD_OK;
    void* d_rows = nullptr;
    void* d_idx = nullptr;
    void* d_vec = nullptr;
    void* d_st = nullptr;
    CUDA_TRY(s, cudaMalloc(&d_rows, nrow * sizeof(FcRow)));
    s->fc_alloc.push_back(d_rows);
    CUDA_TRY(s, cudaMalloc(&d_idx, np * sizeof(int)));
    s->fc_alloc.push_back(d_idx);
    CUDA_TRY(s, cudaMalloc(&d_vec, 9 * nrow * sizeof(double)));  // b, x[2], work[6]
    s->fc_alloc.push_back(d_vec);
    CUDA_TRY(s, cudaMalloc(&d_st, 4 * sizeof(int)));
    s->fc_alloc.push_back(d_st);
    CUDA_TRY(s, cudaMemcpy(d_rows, rows.data(), nrow * sizeof(FcRow), cudaMemcpyHostToDevice));
    CUDA_TRY(s, cudaMemcpy(d_idx, idx.data(), np * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_TRY(s, cudaMemset(d_vec, 0, 9 * nrow * sizeof(double)));
    CUDA_TRY(s, cudaMemset(d_st, 0, 4 * sizeof(int)));
    P.fc_rows = (const FcRow*)d_rows;
    P.fc_idx = (const int*)d_idx;
    P.fc_b = (double*)d_vec;
    P.fc_x = P.fc_b + nrow;
    P.fc_work = P.fc_x + 2 * nrow;
    P.fc_status = (int*)d_st;
    P.fc_n = (int)nrow;
    P.fc_maxit = (int)std::min<long long>(2 * nrow, 1000);
    s->fc_immersed = s->fc_fallback = 0;
    for (const FcRow& r : rows) {
        s->fc_immersed += r.kind == 2;
        s->fc_fallback += r.kind == 3;
    }
    return FDTD_OK;
}

}  // namespace fdtd

extern "C" fdtd_status fdtd_solver_boundary_info(fdtd_solver* s, int64_t* n_rows, int64_t* n_immersed,
                                                 int64_t* n_fallback, int32_t* last_iterations) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    const SolveParams& P = s->hP;
    if (n_rows) *n_rows = P.fc_n;
    if (n_immersed) *n_immersed = s->fc_immersed;
    if (n_fallback) *n_fallback = s->fc_fallback;
    if (last_iterations) {
        *last_iterations = 0;
        if (P.fc_status) {
            CUDA_TRY(s, cudaStreamSynchronize(s->stream));
            CUDA_TRY(s, cudaMemcpy(last_iterations, P.fc_status, sizeof(int32_t), cudaMemcpyDeviceToHost));
        }
    }
    return FDTD_OK;
}
