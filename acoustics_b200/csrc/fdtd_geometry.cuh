// fdtd_geometry.cuh — analytic rigid-body queries, boundary accelerations and
// the weighted least-squares (MLS) solve, shared by host and device code.
//
// These functions are compiled without multiply-add contraction (nvcc
// -fmad=false, host -ffp-contract=off) so that classification, ghost
// pressures and listener samples are reproducible bit for bit between the
// CPU and the GPU.
#pragma once
#include <cfloat>
#include <cmath>

#include "fdtd_device.cuh"

#ifdef __CUDACC__
#define FDTD_HD __host__ __device__ __forceinline__
#else
#define FDTD_HD inline
#endif

namespace fdtd {

constexpr double AABB_CHECK_TOLERANCE_SCALE = 1.1;  // Wavesolver_ConstantsAndTypes.h:78
constexpr double DISTANCE_TOLERANCE = 0.0;          // Wavesolver_ConstantsAndTypes.h:76
constexpr double MLS_FLEISHMAN_RAD = 0.018;         // MLSConstantsAndTypes.h:9

FDTD_HD double dmin(double a, double b) { return a < b ? a : b; }
FDTD_HD double dmax(double a, double b) { return a > b ? a : b; }

// Signed distance of an analytic body, negative inside (stands in for the mesh
// ADF of FDTD_RigidObject::DistanceToMesh, FDTD_RigidObject.cpp:256-277).
FDTD_HD double sdf_local(const DevObject& o, const double p[3]) {
    const double r0 = p[0] - o.c[0], r1 = p[1] - o.c[1], r2 = p[2] - o.c[2];
    if (o.shape == 0) return sqrt(r0 * r0 + r1 * r1 + r2 * r2) - o.size[0];
    double q[3];
    for (int j = 0; j < 3; ++j) q[j] = o.R[0 * 3 + j] * r0 + o.R[1 * 3 + j] * r1 + o.R[2 * 3 + j] * r2;
    if (o.shape == 3) return mesh_sdf(o.mesh, q);
    if (o.shape == 1) {
        double out = 0.0, in = -DBL_MAX;
        for (int j = 0; j < 3; ++j) {
            const double dj = fabs(q[j]) - o.size[j];
            const double m = dj > 0.0 ? dj : 0.0;
            out = out + m * m;
            in = dj > in ? dj : in;
        }
        return sqrt(out) + (in < 0.0 ? in : 0.0);
    }
    double k0 = 0.0, k1 = 0.0;
    for (int j = 0; j < 3; ++j) {
        const double a = q[j] / o.size[j];
        const double b = a / o.size[j];
        k0 = k0 + a * a;
        k1 = k1 + b * b;
    }
    k0 = sqrt(k0);
    k1 = sqrt(k1);
    if (k1 == 0.0) return -dmin(o.size[0], dmin(o.size[1], o.size[2]));
    return k0 * (k0 - 1.0) / k1;
}

// DistanceToMesh with the scaled-AABB early out (FDTD_RigidObject.cpp:259-260,
// FDTD_MovableObject.h:67-73).
FDTD_HD double distance_to_mesh(const DevObject& o, const double p[3]) {
    for (int d = 0; d < 3; ++d) {
        const double sd = o.bdim[d] * AABB_CHECK_TOLERANCE_SCALE;
        if (!(p[d] < (o.bcen[d] + sd) && p[d] > (o.bcen[d] - sd))) return DBL_MAX;
    }
    return sdf_local(o, p);
}

// FDTD_Objects::OccupyByObject (FDTD_Objects.cpp:35-49)
FDTD_HD int occupy_by_object(const SolveParams& P, const double p[3]) {
    for (int o = 0; o < P.n_obj; ++o)
        if (distance_to_mesh(P.obj[o], p) < DISTANCE_TOLERANCE) return o;
    return -1;
}

// FDTD_Objects::OccupyByConstraint + FDTD_PlaneConstraint::Inside (FDTD_PlaneConstraint.h:33-38)
FDTD_HD bool occupy_by_constraint(const SolveParams& P, const double p[3]) {
    for (int i = 0; i < P.n_plane; ++i)
        if ((p[P.plane[i].dir] - P.plane[i].height) * (double)P.plane[i].sign < 0) return true;
    return false;
}

// isFluid lambda of classifyCells_FAST (MAC_Grid.cpp:3566-3577): the centre and
// the six points centre +- h/4 along each axis must be outside every object.
FDTD_HD bool is_fluid(const SolveParams& P, const double pos[3], int& type) {
    bool fluid = !occupy_by_constraint(P, pos) && occupy_by_object(P, pos) < 0;
    for (int d = 0; d < 3 && fluid; ++d) {
        for (int s = -1; s <= 1 && fluid; s += 2) {
            double q[3] = {pos[0], pos[1], pos[2]};
            q[d] = q[d] + (s > 0 ? 1.0 : -1.0) * 0.25 * P.h;
            fluid = occupy_by_object(P, q) < 0;
        }
    }
    if (!fluid) type = occupy_by_constraint(P, pos) ? 1 : 0;
    return fluid;
}

// FDTD_Objects::LowestObjectDistance (FDTD_Objects.cpp:240-257): first object
// with the smallest |distance|; -1 when the scene has no objects.
FDTD_HD int lowest_object(const SolveParams& P, const double p[3], double* distance = nullptr) {
    if (P.n_obj == 0) return -1;
    double dist = DBL_MAX;
    int id = 0;
    for (int o = 0; o < P.n_obj; ++o) {
        const double q = distance_to_mesh(P.obj[o], p);
        if (fabs(q) < fabs(dist)) { dist = q; id = o; }
    }
    if (distance) *distance = dist;
    return id;
}

// FDTD_RigidObject::ReflectAgainstBoundary (FDTD_RigidObject.cpp:429-536, closest
// point branch): bp the closest boundary point, dist the signed distance.
// Outside the body the erected normal is x - bp and the image x + (x - bp);
// inside it is bp - x and the image bp + (bp - x), outside the body.  The
// normal is normalised.  (A box's closest point of an inside point lies on
// the face nearest to it.)
FDTD_HD void reflect_against_boundary(const DevObject& o, const double x[3], double image[3], double bp[3],
                                      double nrm[3], double& dist) {
    const double r[3] = {x[0] - o.c[0], x[1] - o.c[1], x[2] - o.c[2]};
    if (o.shape == 3) {
        // mesh: closest point of the reference's search (FDTD_RigidObject.cpp:453-512;
        // KD_NEAREST_TOLERANCE is 0, so its push-along-the-normal branch never runs)
        double q[3], cpo[3];
        for (int j = 0; j < 3; ++j) q[j] = o.R[0 * 3 + j] * r[0] + o.R[1 * 3 + j] * r[1] + o.R[2 * 3 + j] * r[2];
        int tri = 0;
        dist = mesh_closest_ref(o.mesh, q, cpo, tri);
        for (int i = 0; i < 3; ++i)
            bp[i] = o.c[i] + (o.R[i * 3 + 0] * cpo[0] + o.R[i * 3 + 1] * cpo[1] + o.R[i * 3 + 2] * cpo[2]);
        const double g[3] = {bp[0] - x[0], bp[1] - x[1], bp[2] - x[2]};
        double e[3];
        if (sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) > 1e-10) {  // EPS, config.h:45
            if (dist < 0.0) {
                for (int i = 0; i < 3; ++i) e[i] = bp[i] - x[i];
                for (int i = 0; i < 3; ++i) image[i] = bp[i] + e[i];
            } else {
                for (int i = 0; i < 3; ++i) e[i] = -bp[i] + x[i];
                for (int i = 0; i < 3; ++i) image[i] = x[i] + e[i];
            }
        } else {  // on the triangle: its normal
            const double* n = o.mesh.tris[tri].nf;
            for (int i = 0; i < 3; ++i) e[i] = o.R[i * 3 + 0] * n[0] + o.R[i * 3 + 1] * n[1] + o.R[i * 3 + 2] * n[2];
            for (int i = 0; i < 3; ++i) image[i] = x[i];
        }
        const double en = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        for (int i = 0; i < 3; ++i) nrm[i] = en > 0.0 ? e[i] / en : 0.0;
        return;
    }
    if (o.shape == 0) {
        const double n = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        for (int i = 0; i < 3; ++i) bp[i] = o.c[i] + r[i] / n * o.size[0];
        dist = n - o.size[0];
    } else {
        double q[3], qc[3];
        for (int j = 0; j < 3; ++j) q[j] = o.R[0 * 3 + j] * r[0] + o.R[1 * 3 + j] * r[1] + o.R[2 * 3 + j] * r[2];
        for (int j = 0; j < 3; ++j) qc[j] = dmax(-o.size[j], dmin(o.size[j], q[j]));
        dist = sdf_local(o, x);
        if (dist < 0.0) {  // inside: onto the nearest face
            int jm = 0;
            for (int j = 1; j < 3; ++j)
                if (o.size[j] - fabs(q[j]) < o.size[jm] - fabs(q[jm])) jm = j;
            qc[jm] = q[jm] < 0.0 ? -o.size[jm] : o.size[jm];
        }
        for (int i = 0; i < 3; ++i)
            bp[i] = o.c[i] + (o.R[i * 3 + 0] * qc[0] + o.R[i * 3 + 1] * qc[1] + o.R[i * 3 + 2] * qc[2]);
    }
    double e[3];
    if (dist < 0.0) {
        for (int i = 0; i < 3; ++i) e[i] = bp[i] - x[i];
        for (int i = 0; i < 3; ++i) image[i] = bp[i] + e[i];
    } else {
        for (int i = 0; i < 3; ++i) e[i] = -bp[i] + x[i];
        for (int i = 0; i < 3; ++i) image[i] = x[i] + e[i];
    }
    const double en = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    for (int i = 0; i < 3; ++i) nrm[i] = en > 0.0 ? e[i] / en : 0.0;
}

// ScalarField::enclosingNeighbours (ScalarField.cpp:261-286): up to 8 cells in
// ascending flat-index order; returns the count.
FDTD_HD int enclosing_neighbours(const SolveParams& P, const double x[3], int out[8]) {
    int a0[3], a1[3];
    for (int d = 0; d < 3; ++d) {
        double diff = x[d] - P.bmin[d];
        diff -= P.h / 2.0;
        int i0 = (int)(diff / P.h);
        i0 = i0 < 0 ? 0 : i0;
        i0 = i0 > P.N[d] - 1 ? P.N[d] - 1 : i0;
        a0[d] = i0;
        a1[d] = (diff < 0.0 ? 0 : (i0 + 1 < P.N[d] - 1 ? i0 + 1 : P.N[d] - 1));
    }
    int n = 0;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int l = 0; l < 2; ++l) {
                const int ci = (int)cidx(P, i ? a1[0] : a0[0], j ? a1[1] : a0[1], l ? a1[2] : a0[2]);
                int pos = 0;
                while (pos < n && out[pos] < ci) ++pos;
                if (pos < n && out[pos] == ci) continue;
                for (int q = n; q > pos; --q) out[q] = out[q - 1];
                out[pos] = ci;
                ++n;
            }
    return n;
}

// Boundary acceleration vector of object o at a boundary sample point.
FDTD_HD void boundary_accel(const DevObject& o, const double at[3], double t, double a[3]) {
    a[0] = a[1] = a[2] = 0.0;
    if (o.accel_kind == 0) return;
    const double u = (t - o.t0) / o.tau;
    const double g = o.amp * exp(-(u * u) / 2.0);
    if (o.accel_kind == 1) {
        for (int i = 0; i < 3; ++i) a[i] = o.dir[i] * g;
    } else {
        const double r0 = at[0] - o.c[0], r1 = at[1] - o.c[1], r2 = at[2] - o.c[2];
        const double n = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
        const double r[3] = {r0, r1, r2};
        for (int i = 0; i < 3; ++i) a[i] = (n > 0.0 ? r[i] / n : 0.0) * g;
    }
}

// RASTERIZE ghost-face pressure (MAC_Grid.cpp:1188-1281):
//   pg = p_neig - 0.75 h (grad p . n_cell),  grad p = -rho a(x_face, t),
// for the face owned by a solid cell centred at `owner_pos` whose bulk
// neighbour lies along +-e_dim (sign = topology sign, owner -> neighbour).
FDTD_HD double ghost_pressure(const SolveParams& P, unsigned gobj, const double owner_pos[3], int dim,
                              int sign, double p_neig, double t) {
    if (gobj & GOBJ_CONSTRAINT) return p_neig;
    const unsigned oi = gobj & 0x7F;
    if (oi >= (unsigned)P.n_obj) return p_neig;
    double pos[3] = {owner_pos[0], owner_pos[1], owner_pos[2]};
    pos[dim] += (sign > 0 ? 1.0 : -1.0) * 0.25 * P.h;
    double a[3];
    boundary_accel(P.obj[oi], pos, t, a);
    double g[3];
    for (int i = 0; i < 3; ++i) g[i] = a[i] * (-P.rho);
    double n[3] = {0.0, 0.0, 0.0};
    n[dim] = (sign > 0 ? 1.0 : -1.0);
    const double grad_p_nr = g[0] * n[0] + g[1] * n[1] + g[2] * n[2];
    return p_neig - 0.75 * P.h * grad_p_nr;
}

// Weighted least squares for the constant term of an order-1 MLS fit
// (MLSModeInterpolator::lookup, MLSModeInterpolator.hpp:282-431, weights
// exp(-d^2/(2 r^2)) of :588-598).  Householder QR on the n x 4 weighted
// matrix; A (row-major n x 4) and b are overwritten.  Returns false for a
// rank-deficient stencil.
FDTD_HD bool householder_ls4(double* A, double* b, int n, double& c0) {
    double R[4][4];
    for (int j = 0; j < 4; ++j) {
        double s = 0.0;
        for (int i = j; i < n; ++i) s += A[i * 4 + j] * A[i * 4 + j];
        const double norm = sqrt(s);
        if (!(norm > 0.0)) return false;
        const double x0 = A[j * 4 + j];
        const double alpha = x0 > 0.0 ? -norm : norm;
        A[j * 4 + j] = x0 - alpha;
        double vnorm2 = 0.0;
        for (int i = j; i < n; ++i) vnorm2 += A[i * 4 + j] * A[i * 4 + j];
        for (int cc = j + 1; cc < 4; ++cc) {
            double dot = 0.0;
            for (int i = j; i < n; ++i) dot += A[i * 4 + j] * A[i * 4 + cc];
            const double f = 2.0 * dot / vnorm2;
            for (int i = j; i < n; ++i) A[i * 4 + cc] -= f * A[i * 4 + j];
        }
        {
            double dot = 0.0;
            for (int i = j; i < n; ++i) dot += A[i * 4 + j] * b[i];
            const double f = 2.0 * dot / vnorm2;
            for (int i = j; i < n; ++i) b[i] -= f * A[i * 4 + j];
        }
        R[j][j] = alpha;
        for (int cc = j + 1; cc < 4; ++cc) R[j][cc] = A[j * 4 + cc];
    }
    const double rmax = dmax(dmax(fabs(R[0][0]), fabs(R[1][1])), dmax(fabs(R[2][2]), fabs(R[3][3])));
    for (int j = 0; j < 4; ++j)
        if (fabs(R[j][j]) <= (double)(n > 4 ? n : 4) * 2.220446049250313e-16 * rmax) return false;
    double x[4];
    for (int j = 3; j >= 0; --j) {
        double s = b[j];
        for (int cc = j + 1; cc < 4; ++cc) s -= R[j][cc] * x[cc];
        x[j] = s / R[j][j];
    }
    c0 = x[0];
    return true;
}

// The least-squares solve of householder_ls4 on a fixed block of 8 rows whose
// unused rows are zero (the same minimiser: zero rows change no norm or dot
// product), with every loop unrolled so the block stays in registers.  nk: the
// rows in use, for the rank test.
FDTD_HD bool householder_ls4_rows8(double (&A)[8][4], double (&b)[8], int nk, double& c0) {
    double R[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        double s = 0.0;
#pragma unroll
        for (int i = j; i < 8; ++i) s += A[i][j] * A[i][j];
        const double norm = sqrt(s);
        if (!(norm > 0.0)) return false;
        const double x0 = A[j][j];
        const double alpha = x0 > 0.0 ? -norm : norm;
        A[j][j] = x0 - alpha;
        double vnorm2 = 0.0;
#pragma unroll
        for (int i = j; i < 8; ++i) vnorm2 += A[i][j] * A[i][j];
#pragma unroll
        for (int cc = j + 1; cc < 4; ++cc) {
            double dot = 0.0;
#pragma unroll
            for (int i = j; i < 8; ++i) dot += A[i][j] * A[i][cc];
            const double f = 2.0 * dot / vnorm2;
#pragma unroll
            for (int i = j; i < 8; ++i) A[i][cc] -= f * A[i][j];
        }
        {
            double dot = 0.0;
#pragma unroll
            for (int i = j; i < 8; ++i) dot += A[i][j] * b[i];
            const double f = 2.0 * dot / vnorm2;
#pragma unroll
            for (int i = j; i < 8; ++i) b[i] -= f * A[i][j];
        }
        R[j][j] = alpha;
#pragma unroll
        for (int cc = j + 1; cc < 4; ++cc) R[j][cc] = A[j][cc];
    }
    const double rmax = dmax(dmax(fabs(R[0][0]), fabs(R[1][1])), dmax(fabs(R[2][2]), fabs(R[3][3])));
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (fabs(R[j][j]) <= (double)(nk > 4 ? nk : 4) * 2.220446049250313e-16 * rmax) return false;
    double x[4];
#pragma unroll
    for (int j = 3; j >= 0; --j) {
        double s2 = b[j];
#pragma unroll
        for (int cc = j + 1; cc < 4; ++cc) s2 -= R[j][cc] * x[cc];
        x[j] = s2 / R[j][j];
    }
    c0 = x[0];
    return true;
}

// Fill one weighted MLS row for sample point pt with value val, relative to p.
FDTD_HD void mls_row(const double p[3], const double pt[3], double val, double* Arow, double& b) {
    const double dx = pt[0] - p[0], dy = pt[1] - p[1], dz = pt[2] - p[2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double r2 = MLS_FLEISHMAN_RAD * MLS_FLEISHMAN_RAD;
    const double w = exp(-(d2) / (2. * r2));
    Arow[0] = 1.0 * w;
    Arow[1] = dx * w;
    Arow[2] = dy * w;
    Arow[3] = dz * w;
    b = val * w;
}

}  // namespace fdtd
