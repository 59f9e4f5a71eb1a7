// fdtd_mesh.cuh — rigid bodies given as closed triangle meshes: the distance
// and closest-point queries of FDTD_RigidObject over a bounding-volume
// hierarchy, shared by host and device code (compiled without multiply-add
// contraction, like fdtd_geometry.cuh).
//
// Two queries, as the reference has two:
//   * mesh_sdf: signed distance, negative inside.  The reference reads it from
//     an adaptive distance field built from the mesh (FDTD_RigidObject.cpp:59-76,
//     AdaptiveDistanceField.cpp:70-195: octree of exact closest-point distances,
//     sign from the pseudo-normal of the closest feature [Baerentzen 2002], error
//     tolerance 1e-6 m, Wavesolver_ConstantsAndTypes.h:88-91).  Here: the exact
//     distance to the closest triangle point with the same sign rule.
//   * mesh_closest_ref: TriangleMesh::ComputeClosestPointOnMeshHelper
//     (TriangleMesh.hpp:819-985), the per-triangle projection and barycentric
//     case split of the reference with the sign of the closest triangle's plane
//     side, used by ReflectAgainstBoundary (FDTD_RigidObject.cpp:451-512).  The
//     reference searches the 100 triangles a k-d tree finds nearest; here every
//     triangle is a candidate (the hierarchy prunes exactly).
// Ties (equal squared distance) go to the lowest triangle index, so the result
// does not depend on the traversal order.
#pragma once
#include <cfloat>
#include <climits>
#include <cmath>

#ifdef __CUDACC__
#define FDTD_MHD __host__ __device__ __forceinline__
#else
#define FDTD_MHD inline
#endif

namespace fdtd {

// One triangle in leaf order: vertices (counter-clockwise from outside), its
// index in the mesh, and the pseudo-normals of its face, edges and vertices.
struct MeshTri {
    double p[3][3];
    double nf[3];     // unit face normal
    double ne[3][3];  // edges p0p1, p1p2, p2p0: sum of the two incident unit face normals
    double nv[3][3];  // vertices: angle-weighted sum of the incident unit face normals
    int id;
    int _pad;
};

// Inner node: children first, first + 1 (count == 0).  Leaf: triangles
// [first, first + count).  Boxes are widened a little beyond their triangles,
// so a box is never farther than a triangle inside it after rounding.
struct MeshNode {
    double lo[3], hi[3];
    int first, count;
};

struct MeshView {
    const MeshNode* nodes;
    const MeshTri* tris;
    int n_nodes, n_tris;
};

constexpr int MESH_STACK = 64;  // the host build bounds the depth below this

FDTD_MHD double m_dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

FDTD_MHD double box_dist2(const MeshNode& n, const double q[3]) {
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double e = q[d] < n.lo[d] ? n.lo[d] - q[d] : (q[d] > n.hi[d] ? q[d] - n.hi[d] : 0.0);
        s = s + e * e;
    }
    return s;
}

// Closest point of triangle (a, b, c) to q by its Voronoi regions (Ericson,
// Real-Time Collision Detection, 5.1.5).  region: 0 face, 1 edge ab, 2 edge bc,
// 3 edge ca, 4 vertex a, 5 vertex b, 6 vertex c.
FDTD_MHD void tri_closest_exact(const double q[3], const double a[3], const double b[3], const double c[3],
                                double cp[3], int& region) {
    double ab[3], ac[3], aq[3], bq[3], cq[3];
    for (int i = 0; i < 3; ++i) {
        ab[i] = b[i] - a[i];
        ac[i] = c[i] - a[i];
        aq[i] = q[i] - a[i];
        bq[i] = q[i] - b[i];
        cq[i] = q[i] - c[i];
    }
    const double d1 = m_dot(ab, aq), d2 = m_dot(ac, aq);
    if (d1 <= 0.0 && d2 <= 0.0) {
        for (int i = 0; i < 3; ++i) cp[i] = a[i];
        region = 4;
        return;
    }
    const double d3 = m_dot(ab, bq), d4 = m_dot(ac, bq);
    if (d3 >= 0.0 && d4 <= d3) {
        for (int i = 0; i < 3; ++i) cp[i] = b[i];
        region = 5;
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double v = d1 / (d1 - d3);
        for (int i = 0; i < 3; ++i) cp[i] = a[i] + v * ab[i];
        region = 1;
        return;
    }
    const double d5 = m_dot(ab, cq), d6 = m_dot(ac, cq);
    if (d6 >= 0.0 && d5 <= d6) {
        for (int i = 0; i < 3; ++i) cp[i] = c[i];
        region = 6;
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        for (int i = 0; i < 3; ++i) cp[i] = a[i] + w * ac[i];
        region = 3;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int i = 0; i < 3; ++i) cp[i] = b[i] + w * (c[i] - b[i]);
        region = 2;
        return;
    }
    const double den = 1.0 / (va + vb + vc);
    const double v = vb * den, w = vc * den;
    for (int i = 0; i < 3; ++i) cp[i] = a[i] + ab[i] * v + ac[i] * w;
    region = 0;
}

FDTD_MHD const double* tri_pseudo_normal(const MeshTri& t, int region) {
    if (region == 0) return t.nf;
    if (region <= 3) return t.ne[region - 1];
    return t.nv[region - 4];
}

// TriangleMesh::ComputeClosestPointOnMeshHelper for one triangle
// (TriangleMesh.hpp:835-948): projection onto the plane, barycentric (u, v) of
// the projection, closest point by the seven cases; returns sgn * |q - cp|^2
// with sgn = -1 on the inner side of the plane (t >= 0).
FDTD_MHD double tri_closest_ref(const double q[3], const MeshTri& T, double cp[3]) {
    const double* p0 = T.p[0];
    const double* p1 = T.p[1];
    const double* p2 = T.p[2];
    double e0[3], e1[3];
    for (int i = 0; i < 3; ++i) {
        e0[i] = p2[i] - p0[i];
        e1[i] = p1[i] - p0[i];
    }
    const double dot00 = m_dot(e0, e0), dot01 = m_dot(e0, e1), dot11 = m_dot(e1, e1);
    // n = e1 x e0
    const double n[3] = {e1[1] * e0[2] - e1[2] * e0[1], e1[2] * e0[0] - e1[0] * e0[2], e1[0] * e0[1] - e1[1] * e0[0]};
    const double dpl = n[0] * p0[0] + n[1] * p0[1] + n[2] * p0[2];
    const double t = (dpl - m_dot(n, q)) / m_dot(n, n);
    double pp[3];
    for (int i = 0; i < 3; ++i) pp[i] = q[i] + n[i] * t;
    const double sgn = t >= 0.0 ? -1.0 : 1.0;
    double e2[3];
    for (int i = 0; i < 3; ++i) e2[i] = pp[i] - p0[i];
    const double dot02 = m_dot(e0, e2), dot12 = m_dot(e1, e2);
    const double denom = dot00 * dot11 - dot01 * dot01;
    const double inv = 1. / denom;
    const double u = (dot11 * dot02 - dot01 * dot12) * inv;
    const double v = (dot00 * dot12 - dot01 * dot02) * inv;
    if (u >= 0 && v >= 0 && (u + v) < 1) {
        for (int i = 0; i < 3; ++i) cp[i] = pp[i];
    } else if (u < 0 && v >= 0 && (u + v) < 1) {  // edge p0 p1
        const double l = dot12 > 0.0 ? dot12 : 0.0;
        const double s = dot11;
        for (int i = 0; i < 3; ++i) cp[i] = l > s ? pp[i] + (e1[i] - e2[i]) : pp[i] + (e1[i] * l / s - e2[i]);
    } else if (u >= 0 && v < 0 && (u + v) < 1) {  // edge p0 p2
        const double l = dot02 > 0.0 ? dot02 : 0.0;
        const double s = dot00;
        for (int i = 0; i < 3; ++i) cp[i] = l > s ? pp[i] + (e0[i] - e2[i]) : pp[i] + (e0[i] * l / s - e2[i]);
    } else if (u >= 0 && v >= 0 && (u + v) >= 1) {  // edge p1 p2
        double e12[3], o12[3];
        for (int i = 0; i < 3; ++i) {
            e12[i] = p2[i] - p1[i];
            o12[i] = pp[i] - p1[i];
        }
        const double dl = m_dot(o12, e12);
        const double l = dl > 0.0 ? dl : 0.0;
        const double s = m_dot(e12, e12);
        for (int i = 0; i < 3; ++i) cp[i] = l > s ? pp[i] + (e12[i] - o12[i]) : pp[i] + (e12[i] * l / s - o12[i]);
    } else if (u < 0 && v < 0 && (u + v) < 1) {
        for (int i = 0; i < 3; ++i) cp[i] = p0[i];
    } else if (u < 0 && v >= 0 && (u + v) >= 1) {
        for (int i = 0; i < 3; ++i) cp[i] = p1[i];
    } else if (u >= 0 && v < 0 && (u + v) >= 1) {
        for (int i = 0; i < 3; ++i) cp[i] = p2[i];
    } else {
        // u < 0, v < 0, u + v >= 1 (only through rounding): the nearest vertex to the projection
        double d[3];
        for (int k = 0; k < 3; ++k) {
            const double* pk = T.p[k];
            const double x = pp[0] - pk[0], y = pp[1] - pk[1], z = pp[2] - pk[2];
            d[k] = x * x + y * y + z * z;
        }
        const double* pick = d[0] < d[1] ? (d[0] < d[2] ? p0 : p2) : (d[1] < d[2] ? p1 : p2);
        for (int i = 0; i < 3; ++i) cp[i] = pick[i];
    }
    const double x = q[0] - cp[0], y = q[1] - cp[1], z = q[2] - cp[2];
    return sgn * (x * x + y * y + z * z);
}

// Both queries walk the hierarchy nearer child first and skip a box farther
// than the best squared distance so far (ties are still visited).
// mesh_sdf: exact signed distance (pseudo-normal sign).
FDTD_MHD double mesh_sdf(const MeshView& M, const double q[3]) {
    double best = DBL_MAX, best_s = 0.0;
    int best_id = INT_MAX;
    int stack[MESH_STACK];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const MeshNode& n = M.nodes[stack[--sp]];
        if (box_dist2(n, q) > best) continue;
        if (n.count > 0) {
            for (int k = n.first; k < n.first + n.count; ++k) {
                const MeshTri& T = M.tris[k];
                double cp[3];
                int region;
                tri_closest_exact(q, T.p[0], T.p[1], T.p[2], cp, region);
                const double x = q[0] - cp[0], y = q[1] - cp[1], z = q[2] - cp[2];
                const double d2 = x * x + y * y + z * z;
                if (d2 < best || (d2 == best && T.id < best_id)) {
                    best = d2;
                    best_id = T.id;
                    const double r[3] = {x, y, z};
                    best_s = m_dot(r, tri_pseudo_normal(T, region));
                }
            }
        } else {
            const double dl = box_dist2(M.nodes[n.first], q), dr = box_dist2(M.nodes[n.first + 1], q);
            if (sp + 2 > MESH_STACK) continue;  // the build keeps the depth below MESH_STACK
            if (dl <= dr) {
                stack[sp++] = n.first + 1;
                stack[sp++] = n.first;
            } else {
                stack[sp++] = n.first;
                stack[sp++] = n.first + 1;
            }
        }
    }
    const double d = sqrt(best);
    return best_s < 0.0 ? -d : d;
}

// mesh_closest_ref: signed distance, closest point and closest triangle (its
// index in leaf order) of the reference's closest-point search.
FDTD_MHD double mesh_closest_ref(const MeshView& M, const double q[3], double cp[3], int& tri) {
    double best = DBL_MAX, best_signed = DBL_MAX;
    int best_id = INT_MAX;
    tri = -1;
    int stack[MESH_STACK];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const MeshNode& n = M.nodes[stack[--sp]];
        if (box_dist2(n, q) > best) continue;
        if (n.count > 0) {
            for (int k = n.first; k < n.first + n.count; ++k) {
                const MeshTri& T = M.tris[k];
                double c[3];
                const double ds = tri_closest_ref(q, T, c);
                const double a = fabs(ds);
                if (a < best || (a == best && T.id < best_id)) {
                    best = a;
                    best_signed = ds;
                    best_id = T.id;
                    tri = k;
                    for (int i = 0; i < 3; ++i) cp[i] = c[i];
                }
            }
        } else {
            const double dl = box_dist2(M.nodes[n.first], q), dr = box_dist2(M.nodes[n.first + 1], q);
            if (sp + 2 > MESH_STACK) continue;
            if (dl <= dr) {
                stack[sp++] = n.first + 1;
                stack[sp++] = n.first;
            } else {
                stack[sp++] = n.first;
                stack[sp++] = n.first + 1;
            }
        }
    }
    return best_signed >= 0.0 ? sqrt(best_signed) : -sqrt(-best_signed);
}

}  // namespace fdtd
