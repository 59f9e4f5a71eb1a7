// fdtd_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement (C++/OpenMP) of the reference's collocated FDTD step
// (jhwang7628/acoustics, USE_COLLOCATED, RASTERIZE boundary handling).  It is
// the checker for the CUDA library in acoustics_b200/: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product
// never links, loads or falls back to it.
//
// Parity status: the reference cannot be compiled here (Eigen 3.3.7, Boost,
// libconfig++, libigl absent) and holds no golden vectors, so this
// restatement is "parity unpinned" against the reference binary.  It is pinned
// instead by the reference's own analytic hooks (the acceleration-noise dipole
// sphere, AccelerationNoiseVibrationalSource.cpp:134-162) and by an
// independent numpy restatement on small grids (tests/golden/).
//
// It keeps the reference's data structures where they decide results: three
// rotating pressure buffers, full-grid split pressures and face velocities,
// the PML cell lists with cached coefficients, and the ghost-cell map keyed by
// Szudzik's pairing.  Every function cites the reference file:line it follows.
// Bodies are analytic primitives or closed triangle meshes; mesh queries scan
// every triangle in index order (the library walks a hierarchy over the same
// triangles and breaks ties the same way).
// Compile with -ffp-contract=off so that no multiply-add is fused.

#include "../include/fdtd_c.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double EPS = 1e-10;                       // src/config.h:45
const double DISTANCE_TOLERANCE = 0.0;          // Wavesolver_ConstantsAndTypes.h:76
const double CONDN_LIM = 25.0;                  // Wavesolver_ConstantsAndTypes.h:98
const double GAUSSIAN_CHECK_BOUND = 2.0;        // Wavesolver_ConstantsAndTypes.h:77
const double AABB_CHECK_TOLERANCE_SCALE = 1.1;  // Wavesolver_ConstantsAndTypes.h:78
const double MLS_FLEISHMAN_RAD = 0.018;         // math/MLSConstantsAndTypes.h:9
const double DMAX = std::numeric_limits<double>::max();

struct V3 {
    double v[3];
    V3() : v{0, 0, 0} {}
    V3(double a, double b, double c) : v{a, b, c} {}
    double& operator[](int i) { return v[i]; }
    double operator[](int i) const { return v[i]; }
};

// FDTD_MovableObject::BoundingBox (src/wavesolver/FDTD_MovableObject.h:31-99)
struct OBox {
    V3 mn, mx, dim, cen;
    void Update(const V3& a, const V3& b) {
        mn = a; mx = b;
        for (int d = 0; d < 3; ++d) { dim[d] = mx[d] - mn[d]; cen[d] = (mx[d] + mn[d]) / 2.0; }
    }
    void Union(const OBox& o) {
        for (int d = 0; d < 3; ++d) { mn[d] = std::min(o.mn[d], mn[d]); mx[d] = std::max(o.mx[d], mx[d]); }
        for (int d = 0; d < 3; ++d) { dim[d] = mx[d] - mn[d]; cen[d] = (mx[d] + mn[d]) / 2.0; }
    }
    // Inside(x,y,z,scale), FDTD_MovableObject.h:67-73 (strict)
    bool InsideScaled(const V3& p, double scale) const {
        for (int d = 0; d < 3; ++d) {
            const double sd = dim[d] * scale;
            if (!(p[d] < (cen[d] + sd) && p[d] > (cen[d] - sd))) return false;
        }
        return true;
    }
    // Inside(x,y,z), FDTD_MovableObject.h:61-66 (strict)
    bool Inside(const V3& p) const {
        for (int d = 0; d < 3; ++d)
            if (!(p[d] < mx[d] && p[d] > mn[d])) return false;
        return true;
    }
};

// Closed triangle mesh in its object frame (FDTD_RigidObject::_mesh).  Two
// queries over every triangle in index order (a strict < keeps the first of
// equal squared distances):
//  * Sdf: exact distance to the closest triangle point, signed by the
//    pseudo-normal of the closest feature (face, edge or vertex) as the
//    reference's adaptive distance field signs its samples
//    (AdaptiveDistanceField.cpp:170-195, Baerentzen 2002; its tolerance of 1e-6 m,
//    Wavesolver_ConstantsAndTypes.h:88-91, is what the exact distance stands for);
//  * Closest: TriangleMesh::ComputeClosestPointOnMeshHelper
//    (TriangleMesh.hpp:819-985) over all triangles (the reference's k-d tree
//    hands it the 100 nearest), sign from the closest triangle's plane side.
struct OMesh {
    struct Tri {
        V3 p[3];
        V3 nf;     // unit face normal (p1 - p0) x (p2 - p0)
        V3 ne[3];  // edges p0p1, p1p2, p2p0: sum of the two unit face normals
        V3 nv[3];  // vertices: angle-weighted sum of the unit face normals
    };
    std::vector<Tri> t;
    std::vector<double> verts;

    static double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
    static V3 sub(const V3& a, const V3& b) { return V3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }

    bool build(const fdtd_mesh_desc& m) {
        const int nt = m.n_triangles;
        t.assign(nt, Tri());
        verts.assign(m.vertices, m.vertices + 3 * (size_t)m.n_vertices);
        std::map<std::pair<int, int>, int> edge;  // directed edge -> triangle
        for (int k = 0; k < nt; ++k) {
            for (int j = 0; j < 3; ++j) {
                const int v = m.triangles[3 * k + j];
                t[k].p[j] = V3(m.vertices[3 * v], m.vertices[3 * v + 1], m.vertices[3 * v + 2]);
            }
            const V3 a = sub(t[k].p[1], t[k].p[0]), b = sub(t[k].p[2], t[k].p[0]);
            const V3 n(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
            const double ln = std::sqrt(dot(n, n));
            if (!(ln > 0.0)) return false;
            for (int d = 0; d < 3; ++d) t[k].nf[d] = n[d] / ln;
            for (int j = 0; j < 3; ++j) edge[{m.triangles[3 * k + j], m.triangles[3 * k + (j + 1) % 3]}] = k;
        }
        for (int k = 0; k < nt; ++k)
            for (int j = 0; j < 3; ++j) {
                const auto r = edge.find({m.triangles[3 * k + (j + 1) % 3], m.triangles[3 * k + j]});
                if (r == edge.end()) return false;  // open mesh
                for (int d = 0; d < 3; ++d) t[k].ne[j][d] = t[k].nf[d] + t[r->second].nf[d];
            }
        std::vector<double> vn(verts.size(), 0.0);
        for (int k = 0; k < nt; ++k)
            for (int j = 0; j < 3; ++j) {
                const V3 a = sub(t[k].p[(j + 1) % 3], t[k].p[j]), b = sub(t[k].p[(j + 2) % 3], t[k].p[j]);
                double cs = dot(a, b) / (std::sqrt(dot(a, a)) * std::sqrt(dot(b, b)));
                cs = std::max(-1.0, std::min(1.0, cs));
                const double ang = std::acos(cs);
                const int v = m.triangles[3 * k + j];
                for (int d = 0; d < 3; ++d) vn[3 * v + d] += ang * t[k].nf[d];
            }
        for (int k = 0; k < nt; ++k)
            for (int j = 0; j < 3; ++j) {
                const int v = m.triangles[3 * k + j];
                t[k].nv[j] = V3(vn[3 * v], vn[3 * v + 1], vn[3 * v + 2]);
            }
        return true;
    }

    // closest point of a triangle by its Voronoi regions (Ericson, Real-Time
    // Collision Detection 5.1.5); region 0 face, 1-3 edges p0p1 / p1p2 / p2p0, 4-6 vertices
    static V3 ClosestExact(const V3& q, const Tri& T, int& region) {
        const V3& a = T.p[0];
        const V3& b = T.p[1];
        const V3& c = T.p[2];
        const V3 ab = sub(b, a), ac = sub(c, a), aq = sub(q, a), bq = sub(q, b), cq = sub(q, c);
        const double d1 = dot(ab, aq), d2 = dot(ac, aq);
        if (d1 <= 0.0 && d2 <= 0.0) { region = 4; return a; }
        const double d3 = dot(ab, bq), d4 = dot(ac, bq);
        if (d3 >= 0.0 && d4 <= d3) { region = 5; return b; }
        const double vc = d1 * d4 - d3 * d2;
        if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
            const double v = d1 / (d1 - d3);
            region = 1;
            return V3(a[0] + v * ab[0], a[1] + v * ab[1], a[2] + v * ab[2]);
        }
        const double d5 = dot(ab, cq), d6 = dot(ac, cq);
        if (d6 >= 0.0 && d5 <= d6) { region = 6; return c; }
        const double vb = d5 * d2 - d1 * d6;
        if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
            const double w = d2 / (d2 - d6);
            region = 3;
            return V3(a[0] + w * ac[0], a[1] + w * ac[1], a[2] + w * ac[2]);
        }
        const double va = d3 * d6 - d5 * d4;
        if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
            const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            region = 2;
            return V3(b[0] + w * (c[0] - b[0]), b[1] + w * (c[1] - b[1]), b[2] + w * (c[2] - b[2]));
        }
        const double den = 1.0 / (va + vb + vc);
        const double v = vb * den, w = vc * den;
        region = 0;
        return V3(a[0] + ab[0] * v + ac[0] * w, a[1] + ab[1] * v + ac[1] * w, a[2] + ab[2] * v + ac[2] * w);
    }

    double Sdf(const V3& q) const {
        double best = DMAX, s = 0.0;
        for (const Tri& T : t) {
            int region;
            const V3 cp = ClosestExact(q, T, region);
            const V3 r = sub(q, cp);
            const double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (d2 < best) {
                best = d2;
                const V3& n = region == 0 ? T.nf : (region <= 3 ? T.ne[region - 1] : T.nv[region - 4]);
                s = dot(r, n);
            }
        }
        const double d = std::sqrt(best);
        return s < 0.0 ? -d : d;
    }

    // one triangle of ComputeClosestPointOnMeshHelper (TriangleMesh.hpp:835-948)
    static double ClosestRefTri(const V3& q, const Tri& T, V3& cp) {
        const V3& p0 = T.p[0];
        const V3& p1 = T.p[1];
        const V3& p2 = T.p[2];
        const V3 e0 = sub(p2, p0), e1 = sub(p1, p0);
        const double dot00 = dot(e0, e0), dot01 = dot(e0, e1), dot11 = dot(e1, e1);
        const V3 n(e1[1] * e0[2] - e1[2] * e0[1], e1[2] * e0[0] - e1[0] * e0[2], e1[0] * e0[1] - e1[1] * e0[0]);
        const double dp = n[0] * p0[0] + n[1] * p0[1] + n[2] * p0[2];
        const double tt = (dp - dot(n, q)) / dot(n, n);
        const V3 pp(q[0] + n[0] * tt, q[1] + n[1] * tt, q[2] + n[2] * tt);
        const double sgn = tt >= 0.0 ? -1.0 : 1.0;
        const V3 e2 = sub(pp, p0);
        const double dot02 = dot(e0, e2), dot12 = dot(e1, e2);
        const double denom = dot00 * dot11 - dot01 * dot01;
        const double inv = 1. / denom;
        const double u = (dot11 * dot02 - dot01 * dot12) * inv;
        const double v = (dot00 * dot12 - dot01 * dot02) * inv;
        auto along = [&](const V3& e, const V3& o, double l, double sq) {
            V3 r;
            for (int i = 0; i < 3; ++i) r[i] = l > sq ? pp[i] + (e[i] - o[i]) : pp[i] + (e[i] * l / sq - o[i]);
            return r;
        };
        if (u >= 0 && v >= 0 && (u + v) < 1) cp = pp;
        else if (u < 0 && v >= 0 && (u + v) < 1) cp = along(e1, e2, std::max(dot12, 0.0), dot11);
        else if (u >= 0 && v < 0 && (u + v) < 1) cp = along(e0, e2, std::max(dot02, 0.0), dot00);
        else if (u >= 0 && v >= 0 && (u + v) >= 1) {
            const V3 e12 = sub(p2, p1), o12 = sub(pp, p1);
            cp = along(e12, o12, std::max(dot(o12, e12), 0.0), dot(e12, e12));
        } else if (u < 0 && v < 0 && (u + v) < 1) cp = p0;
        else if (u < 0 && v >= 0 && (u + v) >= 1) cp = p1;
        else if (u >= 0 && v < 0 && (u + v) >= 1) cp = p2;
        else {
            double dd[3];
            for (int k = 0; k < 3; ++k) {
                const V3 r = sub(pp, T.p[k]);
                dd[k] = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            }
            cp = dd[0] < dd[1] ? (dd[0] < dd[2] ? p0 : p2) : (dd[1] < dd[2] ? p1 : p2);
        }
        const V3 r = sub(q, cp);
        return sgn * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    }

    double Closest(const V3& q, V3& cp, int& tri) const {
        double best = DMAX;
        tri = -1;
        for (int k = 0; k < (int)t.size(); ++k) {
            V3 c;
            const double ds = ClosestRefTri(q, t[k], c);
            if (std::fabs(ds) < std::fabs(best)) {
                best = ds;
                tri = k;
                cp = c;
            }
        }
        return best >= 0.0 ? std::sqrt(best) : -std::sqrt(-best);
    }
};

// Quaternion arithmetic of the reference's Quaternion<double> (Quaternion.hpp):
// q = (w, x, y, z); normalize only when |len^2 - 1| > EPS = 1e-12 (:186-195).
struct OQuat {
    double w, x, y, z;
    double LengthSqr() const { return w * w + (x * x + y * y + z * z); }
    void Normalize() {
        double len = LengthSqr();
        if (std::fabs(len - 1.0) > 1e-12) {
            len = 1. / std::sqrt(len);
            w *= len; x *= len; y *= len; z *= len;
        }
    }
    double Dot(const OQuat& b) const { return w * b.w + x * b.x + y * b.y + z * b.z; }
    OQuat Scaled(double s) const { return {w * s, x * s, y * s, z * s}; }
    OQuat Plus(const OQuat& b) const { return {w + b.w, x + b.x, y + b.y, z + b.z}; }
    OQuat Minus(const OQuat& b) const { return {w - b.w, x - b.x, y - b.y, z - b.z}; }
    // Quaternion::slerp, live branch (Quaternion.hpp:392-420)
    OQuat Slerp(double r, const OQuat& q2) const {
        OQuat v0 = *this, v1 = q2;
        v0.Normalize();
        v1.Normalize();
        double dot = v0.Dot(v1);
        if (std::fabs(dot) > 0.9995) {
            OQuat ret = v0.Plus(v1.Minus(v0).Scaled(r));
            ret.Normalize();
            return ret;
        }
        if (dot < 0.0) { v1 = v1.Scaled(-1.0); dot = -dot; }
        dot = std::min(std::max(dot, -1.0), 1.0);
        const double theta_0 = std::acos(dot);
        const double theta = theta_0 * r;
        OQuat v2 = v1.Minus(v0.Scaled(dot));
        v2.Normalize();
        return v0.Scaled(std::cos(theta)).Plus(v2.Scaled(std::sin(theta)));
    }
};

// Rigid object: an analytic body standing in for FDTD_RigidObject's mesh + ADF
// (FDTD_RigidObject.cpp:256-277), or a triangle mesh; negative inside.
struct Obj {
    fdtd_object_desc d;
    V3 c;        // current centre
    OBox box;    // _bboxWorld
    OBox ubox;   // _bboxWorldUnion2Steps
    const OMesh* mesh = nullptr;
    V3 mlo, mhi;  // mesh: extent of rotation * v
    // keyframed motion: frames (centre, quaternion) every kf_step seconds, rest rotation R0
    std::vector<double> kf;
    double kf_step = 0;
    double R0[9];

    void MeshExtent() {
        if (!mesh) return;
        const std::vector<double>& v = mesh->verts;
        for (int d = 0; d < 3; ++d) { mlo[d] = DMAX; mhi[d] = -DMAX; }
        for (size_t k = 0; k + 2 < v.size(); k += 3)
            for (int d = 0; d < 3; ++d) {
                const double w = d_rot(d, 0) * v[k] + d_rot(d, 1) * v[k + 1] + d_rot(d, 2) * v[k + 2];
                mlo[d] = std::min(mlo[d], w);
                mhi[d] = std::max(mhi[d], w);
            }
    }
    double d_rot(int i, int j) const { return d.rotation[i * 3 + j]; }

    // FDTD_RigidObject_Blender_Animator::GetRigidObjectTransform (FDTD_RigidObject_Animator.cpp:128-155),
    // start time 0; then AnimateObjects' normalize (FDTD_Objects.cpp:577) and
    // SetRigidBodyTransform's axis-angle rotation (FDTD_RigidObject.cpp:549-566)
    void KeyframePose(double time) {
        const int n = (int)(kf.size() / 7);
        const double u = time / kf_step;
        int idx_0 = 0;
        if (u > 0) idx_0 = u >= (double)n ? n - 1 : (int)u;
        idx_0 = std::min(std::max(0, idx_0), n - 1);
        const int idx_1 = std::min(idx_0 + 1, n - 1);
        const double t_0 = idx_0 * kf_step, t_1 = idx_1 * kf_step;
        const double alpha = (idx_0 == idx_1 ? 1.0 : (time - t_0) / (t_1 - t_0));
        const double* a = &kf[7 * (size_t)idx_0];
        const double* b = &kf[7 * (size_t)idx_1];
        for (int k = 0; k < 3; ++k) c[k] = a[k] * (1.0 - alpha) + b[k] * alpha;
        OQuat q = OQuat{a[3], a[4], a[5], a[6]}.Slerp(alpha, OQuat{b[3], b[4], b[5], b[6]});
        q.Normalize();
        // Quaternion::toAxisRotR (Quaternion.hpp:298-313)
        const double rad = 2.0 * std::acos(q.w);
        double ax = 0.0, ay = 1.0, az = 0.0;
        if (!(rad < 1e-12)) {
            ax = q.x; ay = q.y; az = q.z;
            const double l = std::sqrt(ax * ax + ay * ay + az * az);
            if (l > 0) { ax /= l; ay /= l; az /= l; }
        }
        // the axis-angle matrix (Rodrigues), grouped as AngleAxis::toRotationMatrix
        const double sn = std::sin(rad), cs = std::cos(rad);
        const double sx = sn * ax, sy = sn * ay, sz = sn * az;
        const double cx = (1.0 - cs) * ax, cy = (1.0 - cs) * ay, cz = (1.0 - cs) * az;
        double R[9];
        R[1] = cx * ay - sz; R[3] = cx * ay + sz;
        R[2] = cx * az + sy; R[6] = cx * az - sy;
        R[5] = cy * az - sx; R[7] = cy * az + sx;
        R[0] = cx * ax + cs; R[4] = cy * ay + cs; R[8] = cz * az + cs;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                d.rotation[i * 3 + j] = R[i * 3 + 0] * R0[0 * 3 + j] + R[i * 3 + 1] * R0[1 * 3 + j] + R[i * 3 + 2] * R0[2 * 3 + j];
        MeshExtent();
    }

    void pose(double t) {  // ballistic kinematics x(t) = x0 + v t + g t^2/2
        if (d.motion == FDTD_MOTION_KEYFRAMED) { KeyframePose(t); return; }
        for (int a = 0; a < 3; ++a) {
            if (d.motion == FDTD_MOTION_BALLISTIC)
                c[a] = d.center[a] + d.velocity[a] * t + 0.5 * d.gravity[a] * t * t;
            else
                c[a] = d.center[a];
        }
    }
    V3 half_extent() const {
        V3 e;
        for (int i = 0; i < 3; ++i) {
            if (d.shape == FDTD_SHAPE_SPHERE) { e[i] = d.size[0]; continue; }
            double s = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double rij = d.rotation[i * 3 + j];
                if (d.shape == FDTD_SHAPE_BOX) s = s + std::fabs(rij) * d.size[j];
                else s = s + (rij * d.size[j]) * (rij * d.size[j]);
            }
            e[i] = (d.shape == FDTD_SHAPE_BOX) ? s : std::sqrt(s);
        }
        return e;
    }
    // FDTD_RigidObject::UpdateBoundingBox (FDTD_RigidObject.cpp:190-226)
    void UpdateBoundingBox() {
        ubox = box;
        V3 e = half_extent(), a, b;
        for (int i = 0; i < 3; ++i) { a[i] = c[i] - e[i]; b[i] = c[i] + e[i]; }
        if (mesh)
            for (int i = 0; i < 3; ++i) { a[i] = c[i] + mlo[i]; b[i] = c[i] + mhi[i]; }
        box.Update(a, b);
        ubox.Union(box);
    }
    void ResetUnionBox() { ubox = box; }

    double sdf_local(const V3& p) const {
        V3 r;
        for (int a = 0; a < 3; ++a) r[a] = p[a] - c[a];
        if (d.shape == FDTD_SHAPE_SPHERE)
            return std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) - d.size[0];
        V3 q;  // object frame: R^T r
        for (int j = 0; j < 3; ++j)
            q[j] = d.rotation[0 * 3 + j] * r[0] + d.rotation[1 * 3 + j] * r[1] + d.rotation[2 * 3 + j] * r[2];
        if (mesh) return mesh->Sdf(q);
        if (d.shape == FDTD_SHAPE_BOX) {
            double out = 0.0, in = -DMAX;
            for (int j = 0; j < 3; ++j) {
                const double dj = std::fabs(q[j]) - d.size[j];
                const double m = dj > 0.0 ? dj : 0.0;
                out = out + m * m;
                in = dj > in ? dj : in;
            }
            return std::sqrt(out) + (in < 0.0 ? in : 0.0);
        }
        // ellipsoid: first-order distance estimate k0*(k0-1)/k1, exact sign
        double k0 = 0.0, k1 = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double a = q[j] / d.size[j];
            const double b = a / d.size[j];
            k0 = k0 + a * a;
            k1 = k1 + b * b;
        }
        k0 = std::sqrt(k0);
        k1 = std::sqrt(k1);
        if (k1 == 0.0) return -std::min(d.size[0], std::min(d.size[1], d.size[2]));
        return k0 * (k0 - 1.0) / k1;
    }
    // DistanceToMesh with the scaled-AABB early out (FDTD_RigidObject.cpp:256-277)
    double DistanceToMesh(const V3& p) const {
        if (!box.InsideScaled(p, AABB_CHECK_TOLERANCE_SCALE)) return DMAX;
        return sdf_local(p);
    }
    // boundary acceleration vector at a boundary sample point
    V3 accel(const V3& at, double t) const {
        V3 a;
        if (d.accel_kind == FDTD_ACCEL_NONE) return a;
        const double u = (t - d.accel_t0) / d.accel_tau;
        const double g = d.accel_amplitude * std::exp(-(u * u) / 2.0);
        if (d.accel_kind == FDTD_ACCEL_GAUSSIAN_TRANSLATION) {
            for (int i = 0; i < 3; ++i) a[i] = d.accel_dir[i] * g;
        } else {  // pulsation: along the outward radial direction of the sphere
            V3 r;
            for (int i = 0; i < 3; ++i) r[i] = at[i] - c[i];
            const double n = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (int i = 0; i < 3; ++i) a[i] = (n > 0.0 ? r[i] / n : 0.0) * g;
        }
        return a;
    }
    // ReflectAgainstBoundary (FDTD_RigidObject.cpp:429-536), closest-point branch:
    // outside, erected normal x - bp and image x + (x - bp); inside, normal bp - x
    // and image bp + (bp - x) (the mirror point outside the body).
    void Reflect(const V3& x, V3& image, V3& bp, V3& nrm, double& dist) const {
        V3 r;
        for (int i = 0; i < 3; ++i) r[i] = x[i] - c[i];
        if (mesh) {
            // FDTD_RigidObject.cpp:453-512 (KD_NEAREST_TOLERANCE = 0: no push along the normal)
            V3 q, cpo;
            for (int j = 0; j < 3; ++j)
                q[j] = d.rotation[0 * 3 + j] * r[0] + d.rotation[1 * 3 + j] * r[1] + d.rotation[2 * 3 + j] * r[2];
            int tri = 0;
            dist = mesh->Closest(q, cpo, tri);
            for (int i = 0; i < 3; ++i)
                bp[i] = c[i] + (d.rotation[i * 3 + 0] * cpo[0] + d.rotation[i * 3 + 1] * cpo[1] + d.rotation[i * 3 + 2] * cpo[2]);
            const V3 g(bp[0] - x[0], bp[1] - x[1], bp[2] - x[2]);
            V3 e;
            if (std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) > 1e-10) {  // EPS, config.h:45
                const bool in = dist < 0.0;
                for (int i = 0; i < 3; ++i) e[i] = in ? bp[i] - x[i] : -bp[i] + x[i];
                for (int i = 0; i < 3; ++i) image[i] = in ? bp[i] + e[i] : x[i] + e[i];
            } else {
                const V3& n = mesh->t[tri].nf;
                for (int i = 0; i < 3; ++i)
                    e[i] = d.rotation[i * 3 + 0] * n[0] + d.rotation[i * 3 + 1] * n[1] + d.rotation[i * 3 + 2] * n[2];
                image = x;
            }
            const double en = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            for (int i = 0; i < 3; ++i) nrm[i] = en > 0.0 ? e[i] / en : 0.0;
            return;
        }
        if (d.shape == FDTD_SHAPE_SPHERE) {
            const double n = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (int i = 0; i < 3; ++i) bp[i] = c[i] + r[i] / n * d.size[0];
            dist = n - d.size[0];
        } else {  // box (axis frame via rotation)
            V3 q, qc;
            for (int j = 0; j < 3; ++j)
                q[j] = d.rotation[0 * 3 + j] * r[0] + d.rotation[1 * 3 + j] * r[1] + d.rotation[2 * 3 + j] * r[2];
            dist = sdf_local(x);
            if (dist >= 0.0) {  // outside: clamp onto the box
                for (int j = 0; j < 3; ++j) qc[j] = std::max(-d.size[j], std::min(d.size[j], q[j]));
            } else {  // inside: the nearest face
                int best = 0;
                double gap = d.size[0] - std::fabs(q[0]);
                for (int j = 1; j < 3; ++j)
                    if (d.size[j] - std::fabs(q[j]) < gap) {
                        gap = d.size[j] - std::fabs(q[j]);
                        best = j;
                    }
                qc = q;
                qc[best] = q[best] < 0.0 ? -d.size[best] : d.size[best];
            }
            for (int i = 0; i < 3; ++i)
                bp[i] = c[i] + (d.rotation[i * 3 + 0] * qc[0] + d.rotation[i * 3 + 1] * qc[1] + d.rotation[i * 3 + 2] * qc[2]);
        }
        V3 e;
        const bool inside = dist < 0.0;
        for (int i = 0; i < 3; ++i) e[i] = inside ? bp[i] - x[i] : x[i] - bp[i];
        for (int i = 0; i < 3; ++i) image[i] = inside ? bp[i] + e[i] : x[i] + e[i];
        const double en = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        for (int i = 0; i < 3; ++i) nrm[i] = en > 0.0 ? e[i] / en : 0.0;
    }
};

// MAC_Grid::GhostCell (MAC_Grid.h:97-145)
struct GhostCell {
    int owner, neighbour, topology, type;
    int boundaryObject = -1;
    double distance = DMAX;
    V3 position;
    double pressure = 0.0;
};
using Key = unsigned long long;
// Szudzik pairing, MAC_Grid.h:108-116
inline Key MakeKey(int a_, int b_) {
    const unsigned long long a = std::min(a_, b_);
    const unsigned long long b = std::max(a_, b_);
    return (a >= b ? a * a + a + b : a + b * b);
}

// MAC_Grid::PML_PressureCell / PML_VelocityCell (MAC_Grid.h:233-259)
struct PMLPCell { int index; int vl[3], vr[3]; double upd[3], div[3]; };
struct PMLVCell { int index, dim, pl, pr; double upd, grad; };

struct Oracle {
    // settings
    double h, c, rho, k, alpha;
    double absorptionWidth, absorptionStrength;
    int preset;
    bool fullyCoupled = false;  // boundaryHandlingType (ImpulseResponseParser.cpp:547-555)
    int fcIterations = 0;       // BiCGSTAB iterations of the last FULLY_COUPLED solve
    bool engquistMissingGhost = false;  // an Engquist stencil met a ghost cell without a face record
    double endTime;
    // pressure field (ScalarField, ScalarField.cpp:29-50)
    int N[3];
    V3 bmin, bmax;
    int ncell;
    int vN[3][3];  // velocity grid divisions
    V3 vmin[3];
    // objects, constraints, sources, listeners
    std::vector<OMesh> meshes;  // before objs: objects point into it
    std::vector<Obj> objs;
    std::vector<fdtd_plane_desc> planes;
    std::vector<fdtd_gaussian_source_desc> srcs;
    std::vector<OBox> srcBox;
    std::vector<V3> listeners;
    // state (PML_WaveSolver.h:65-80)
    std::vector<double> pCol[3];
    int pColInd = 1;
    std::vector<double> lap[2];
    int lapInd = 1;
    std::vector<double> pDir[3];
    std::vector<double> vel[3];
    double currentTime = 0.0, stateTime = 0.0;
    long long timeIndex = 0;
    // classification (MAC_Grid.h)
    std::vector<char> isBulk, isGhost, isPML, isCavity, validHistory;
    std::vector<char> gcTypeOf;  // constraint flag of solid cells
    std::map<Key, GhostCell> ghosts;
    std::map<int, std::set<Key>> ghostTree;
    std::vector<PMLPCell> pmlP;
    std::vector<PMLVCell> pmlV;
    std::string err;

    // ----- ScalarField helpers (ScalarField.cpp:86-140) -----
    int cellIndex(int i, int j, int l) const { return i * (N[1] * N[2]) + j * N[2] + l; }
    void cellIJK(int f, int ijk[3]) const {
        ijk[0] = f / (N[1] * N[2]);
        f -= ijk[0] * (N[1] * N[2]);
        ijk[1] = f / N[2];
        f -= ijk[1] * N[2];
        ijk[2] = f;
    }
    V3 cellPosition(int f) const {
        int ijk[3];
        cellIJK(f, ijk);
        V3 p;
        for (int d = 0; d < 3; ++d) { p[d] = bmin[d]; p[d] += (0.5 + (double)ijk[d]) * h; }
        return p;
    }
    int vIndex(int dim, int i, int j, int l) const { return i * (vN[dim][1] * vN[dim][2]) + j * vN[dim][2] + l; }
    V3 vPosition(int dim, int i, int j, int l) const {
        const int ijk[3] = {i, j, l};
        V3 p;
        for (int d = 0; d < 3; ++d) { p[d] = vmin[dim][d]; p[d] += (0.5 + (double)ijk[d]) * h; }
        return p;
    }

    // MAC_Grid::InsidePML (MAC_Grid.cpp:4027-4062).  Preset 0: PML on every
    // side; 1: on the low sides and +y (walls +x, +z); 2: on +z only.
    bool InsidePML(const V3& x) const {
        const double pmlWidth = absorptionWidth + 1E-12;
        for (int d = 0; d < 3; ++d) {
            const double hMin = x[d] - bmin[d];
            const double hMax = bmax[d] - x[d];
            if (preset == 0) {
                if (hMin <= pmlWidth) return true;
                if (hMax <= pmlWidth) return true;
            } else if (preset == 1) {
                if (hMin <= pmlWidth || (d == 1 && hMax <= pmlWidth)) return true;
            } else if (preset == 2) {
                if (d == 2 && hMax <= pmlWidth) return true;
            }
        }
        return false;
    }
    // MAC_Grid::PML_absorptionCoefficient, quadratic profile (MAC_Grid.cpp:4064-4101).
    // pow(x,2) is folded to x*x by the compiler without fast-math; written out here.
    double PML_absorptionCoefficient(const V3& x, int d) const {
        const double w = absorptionWidth;
        const double hMin = x[d] - bmin[d];
        const double hMax = bmax[d] - x[d];
        const double a2 = w * w;
        const double distMin = w - hMin;
        const double distMax = w - hMax;
        if (preset == 0) {
            if (hMin <= w) return absorptionStrength * (distMin * distMin) / a2;
            if (hMax <= w) return absorptionStrength * (distMax * distMax) / a2;
        } else if (preset == 1) {
            if (hMin <= w) return absorptionStrength * (distMin * distMin) / a2;
            if (d == 1 && hMax <= w) return absorptionStrength * (distMax * distMax) / a2;
        } else if (preset == 2) {
            if (d != 2 || hMin <= w) return 0.0;
            if (hMax <= w) return absorptionStrength * (distMax * distMax) / a2;
        }
        return 0.0;
    }
    // ScalarField::boundaryCellNormal (ScalarField.h:202-213): -1 / +1 where the
    // cell sits `off` cells from the low / high side of an axis
    void boundaryCellNormal(const int ijk[3], int off, int n[3]) const {
        for (int d = 0; d < 3; ++d) n[d] = ijk[d] == off ? -1 : (ijk[d] == N[d] - 1 - off ? 1 : 0);
    }
    // ScalarField::cellIndex(d0, d1, d2, i0, i1, i2): indices given per permuted axis
    int cellIndexP(int d0, int d1, int d2, int i0, int i1, int i2) const {
        int a[3];
        a[d0] = i0;
        a[d1] = i1;
        a[d2] = i2;
        return cellIndex(a[0], a[1], a[2]);
    }

    // ----- objects (FDTD_Objects.cpp) -----
    // OccupyByObject (FDTD_Objects.cpp:35-49): first object (ascending id) with d < 0
    int OccupyByObject(const V3& p) const {
        for (size_t o = 0; o < objs.size(); ++o)
            if (objs[o].DistanceToMesh(p) < DISTANCE_TOLERANCE) return (int)o;
        return -1;
    }
    // OccupyByConstraint (FDTD_Objects.cpp:53-72) + FDTD_PlaneConstraint::Inside
    bool OccupyByConstraint(const V3& p) const {
        for (const auto& pl : planes)
            if ((p[pl.normal_dir] - pl.height) * (double)pl.normal_sign < 0) return true;
        return false;
    }
    // LowestObjectDistance (FDTD_Objects.cpp:240-257)
    void LowestObjectDistance(const V3& p, double& distance, int& objectID) const {
        if (objs.empty()) return;  // returns false, outputs untouched
        distance = DMAX;
        objectID = 0;
        for (size_t o = 0; o < objs.size(); ++o) {
            const double q = objs[o].DistanceToMesh(p);
            if (std::fabs(q) < std::fabs(distance)) { distance = q; objectID = (int)o; }
        }
    }
    // isFluid lambda (MAC_Grid.cpp:3566-3577): centre and +-h/4 along each axis
    bool isFluid(const V3& pos, int& type) const {
        bool fluid = !OccupyByConstraint(pos) && OccupyByObject(pos) < 0;
        for (int d = 0; d < 3 && fluid; ++d) {
            for (int s = -1; s <= 1 && fluid; s += 2) {
                V3 q = pos;
                q[d] = q[d] + (s > 0 ? 1.0 : -1.0) * 0.25 * h;
                fluid = OccupyByObject(q) < 0;
            }
        }
        if (!fluid) type = OccupyByConstraint(pos) ? 1 : 0;
        return fluid;
    }

    // ScalarField::GetIterationBox (ScalarField.cpp:288-314)
    void GetIterationBox(V3 mn, V3 mx, int start[3], int range[3]) const {
        auto inside = [&](const V3& x) {
            return x[0] >= bmin[0] && x[1] >= bmin[1] && x[2] >= bmin[2] && x[0] <= bmax[0] &&
                   x[1] <= bmax[1] && x[2] <= bmax[2];
        };
        const V3 imn = mn, imx = mx;
        if (!inside(imn)) for (int d = 0; d < 3; ++d) mn[d] = std::max(bmin[d], mn[d]);
        if (!inside(imx)) for (int d = 0; d < 3; ++d) mx[d] = std::min(bmax[d], mx[d]);
        for (int d = 0; d < 3; ++d) {
            start[d] = (int)std::floor((mn[d] - bmin[d]) / h);
            const int end = (int)std::ceil((mx[d] - bmin[d]) / h);
            range[d] = std::max(end - start[d], 1);
            // the reference indexes out of range when a box leaves the grid; clamp
            if (start[d] < 0) { range[d] += start[d]; start[d] = 0; }
            if (start[d] + range[d] > N[d]) range[d] = N[d] - start[d];
            if (range[d] < 0) range[d] = 0;
        }
    }

    // MAC_Grid::classifyCells_FAST (MAC_Grid.cpp:3455-3891), rigid objects and planes only
    void classifyCells_FAST() {
        std::copy(isBulk.begin(), isBulk.end(), validHistory.begin());
        std::fill(isBulk.begin(), isBulk.end(), 1);
        std::fill(isCavity.begin(), isCavity.end(), 0);
        std::fill(isGhost.begin(), isGhost.end(), 0);
        std::fill(gcTypeOf.begin(), gcTypeOf.end(), 0);
        std::vector<char> classified(ncell, 0);
        ghosts.clear();

        std::vector<std::pair<std::vector<int>, std::vector<int>>> boxes;  // start, range
        for (const auto& o : objs) {
            V3 mx = o.ubox.mx, mn = o.ubox.mn;
            for (const auto& pl : planes) {
                if (pl.normal_sign > 0) mn[pl.normal_dir] = std::max(mn[pl.normal_dir], pl.height);
                else mx[pl.normal_dir] = std::min(mx[pl.normal_dir], pl.height);
            }
            int s[3], r[3];
            GetIterationBox(mn, mx, s, r);
            boxes.push_back({{s[0], s[1], s[2]}, {r[0], r[1], r[2]}});
        }
        for (const auto& pl : planes) {
            const double NEG_INF = std::numeric_limits<double>::lowest();
            V3 mn(NEG_INF, NEG_INF, NEG_INF), mx(DMAX, DMAX, DMAX);
            if (pl.normal_sign > 0) mx[pl.normal_dir] = pl.height;
            else mn[pl.normal_dir] = pl.height;
            int s[3], r[3];
            GetIterationBox(mn, mx, s, r);
            boxes.push_back({{s[0], s[1], s[2]}, {r[0], r[1], r[2]}});
        }
        std::vector<int> candidates;
        for (const auto& b : boxes) {
            const int* s = b.first.data();
            const int* r = b.second.data();
            const long total = (long)r[0] * r[1] * r[2];
            std::vector<char> solid(total, 0), type(total, 0);
#pragma omp parallel for schedule(static)
            for (long t = 0; t < total; ++t) {
                const int ii = s[0] + (int)(t / ((long)r[1] * r[2]));
                const int jj = s[1] + (int)((t / r[2]) % r[1]);
                const int kk = s[2] + (int)(t % r[2]);
                const int ci = cellIndex(ii, jj, kk);
                if (classified[ci]) continue;
                int ty = 0;
                if (!isFluid(cellPosition(ci), ty)) { solid[t] = 1; type[t] = (char)ty; }
            }
            for (long t = 0; t < total; ++t) {
                const int ii = s[0] + (int)(t / ((long)r[1] * r[2]));
                const int jj = s[1] + (int)((t / r[2]) % r[1]);
                const int kk = s[2] + (int)(t % r[2]);
                const int ci = cellIndex(ii, jj, kk);
                if (classified[ci]) continue;
                if (solid[t]) { isBulk[ci] = 0; gcTypeOf[ci] = type[t]; candidates.push_back(ci); }
                classified[ci] = 1;
            }
        }
        // ghost faces of every solid candidate (MAC_Grid.cpp:3790-3880)
        for (int ci : candidates) {
            pCol[0][ci] = 0.0;
            pCol[1][ci] = 0.0;
            pCol[2][ci] = 0.0;
            int ijk[3];
            cellIJK(ci, ijk);
            bool is_ghost = false;
            for (int dim = 0; dim < 3; ++dim) {
                for (int idx = -1; idx <= 1; idx += 2) {  // ScalarField::cellNeighbours order
                    int n[3] = {ijk[0], ijk[1], ijk[2]};
                    n[dim] += idx;
                    if (n[dim] < 0 || n[dim] >= N[dim]) continue;
                    const int ns = cellIndex(n[0], n[1], n[2]);
                    if (!isBulk[ns]) continue;
                    is_ghost = true;
                    GhostCell gc;  // MakeGhostCell (MAC_Grid.cpp:4310-4340)
                    gc.owner = ci;
                    gc.neighbour = ns;
                    gc.topology = idx * (dim + 1);
                    gc.type = gcTypeOf[ci];
                    gc.position = cellPosition(ci);
                    gc.position[dim] += (gc.topology > 0 ? 1.0 : -1.0) * 0.25 * h;
                    LowestObjectDistance(cellPosition(ci), gc.distance, gc.boundaryObject);
                    ghosts[MakeKey(ci, ns)] = gc;
                }
            }
            isGhost[ci] = is_ghost;
        }
        ghostTree.clear();
        for (auto& m : ghosts) ghostTree[m.second.owner].insert(m.first);
    }

    // MAC_Grid::classifyCells PML part (MAC_Grid.cpp:2397-2693); no boundary
    // fields are registered by the settings-based constructor, so every cell is
    // bulk at this point and the lists cover the whole PML shell.
    void classifyPML() {
        pmlP.clear();
        pmlV.clear();
        std::fill(isPML.begin(), isPML.end(), 0);
        for (int ci = 0; ci < ncell; ++ci) {
            const V3 pos = cellPosition(ci);
            if (!InsidePML(pos)) continue;
            PMLPCell cell;
            cell.index = ci;
            int ijk[3];
            cellIJK(ci, ijk);
            for (int dim = 0; dim < 3; ++dim) {
                const double sigma = PML_absorptionCoefficient(pos, dim);
                const double directional = 1.0 / k + sigma / 2.0;          // MAC_Grid.h:550-553
                cell.upd[dim] = (1.0 / k - sigma / 2.0) / directional;      // MAC_Grid.h:558-561
                cell.div[dim] = (-1.0 * rho * c * c / directional);         // MAC_Grid.h:566-569
                int a[3] = {ijk[0], ijk[1], ijk[2]};
                cell.vl[dim] = vIndex(dim, a[0], a[1], a[2]);
                a[dim] += 1;
                cell.vr[dim] = vIndex(dim, a[0], a[1], a[2]);
            }
            pmlP.push_back(cell);
            isPML[ci] = 1;
        }
        for (int dim = 0; dim < 3; ++dim) {
            for (int i = 0; i < vN[dim][0]; ++i)
                for (int j = 0; j < vN[dim][1]; ++j)
                    for (int l = 0; l < vN[dim][2]; ++l) {
                        const int ijk[3] = {i, j, l};
                        if (ijk[dim] == 0 || ijk[dim] == vN[dim][dim] - 1) continue;  // rigid outer wall
                        const V3 pos = vPosition(dim, i, j, l);
                        if (!InsidePML(pos)) continue;
                        const double sigma = PML_absorptionCoefficient(pos, dim);
                        PMLVCell v;
                        v.index = vIndex(dim, i, j, l);
                        v.dim = dim;
                        double u = 1.0 / k - sigma / 2.0;   // MAC_Grid.h:530-536
                        u /= 1.0 / k + sigma / 2.0;
                        v.upd = u;
                        double g = 1.0 / k + sigma / 2.0;   // MAC_Grid.h:541-547
                        g *= rho * h;
                        v.grad = -1.0 / g;
                        int a[3] = {i, j, l};
                        v.pr = cellIndex(a[0], a[1], a[2]);
                        a[dim] -= 1;
                        v.pl = cellIndex(a[0], a[1], a[2]);
                        pmlV.push_back(v);
                    }
        }
    }

    // GaussianPressureSource::Evaluate, USE_COLLOCATED (GaussianPressureSource.cpp:6-30)
    double EvaluatePressureSources(const V3& x, double t) const {
        double value_sum = 0;
        for (size_t s = 0; s < srcs.size(); ++s) {
            const OBox& bb = srcBox[s];
            double v = 0.0;
            if (bb.Inside(x)) {
                const V3& sp = bb.cen;
                v = (x[0] - sp[0]) * (x[0] - sp[0]) + (x[1] - sp[1]) * (x[1] - sp[1]) +
                    (x[2] - sp[2]) * (x[2] - sp[2]);
                v = -v / (2.0 * srcs[s].width_space * srcs[s].width_space);
                v = std::exp(v);
                const double u = (t - srcs[s].offset_time) / srcs[s].width_time;
                v *= std::exp(-(u * u) / 2.0);
                v *= 1. / 3.6836 * srcs[s].normalize_constant;
            }
            value_sum += v;
        }
        return value_sum;
    }

    // MAC_Grid::PML_pressureUpdateGhostCells, RASTERIZE (MAC_Grid.cpp:1131-1310).
    // With RASTERIZE every row of the sparse system is the identity and Eigen's
    // BiCGSTAB returns the right-hand side exactly, so gc.pressure = pg.
    void PML_pressureUpdateGhostCells(const std::vector<double>& p, double t) {
        std::vector<GhostCell*> list;
        list.reserve(ghosts.size());
        for (auto& m : ghosts) list.push_back(&m.second);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)list.size(); ++i) {
            GhostCell& gc = *list[i];
            const double p_neig = p[gc.neighbour];
            if (gc.type == 1) { gc.pressure = p_neig; continue; }
            const Obj& o = objs[gc.boundaryObject];
            const V3 a = o.accel(gc.position, t);
            V3 grad_p;
            for (int d = 0; d < 3; ++d) grad_p[d] = a[d] * (-rho);
            V3 n;
            n[std::abs(gc.topology) - 1] = (gc.topology > 0 ? 1.0 : -1.0);
            const double grad_p_nr = grad_p[0] * n[0] + grad_p[1] * n[1] + grad_p[2] * n[2];
            gc.pressure = p_neig - 0.75 * h * grad_p_nr;
        }
    }

    // ----- FULLY_COUPLED ghost cells (MAC_Grid.cpp:1131-1425, use_immerse_interface) -----
    // Trilinear Vandermonde rows in the scaled coordinates of FillVandermonde*S
    // (MAC_Grid.cpp:4444-4510).
    static void vdmRegular(const V3& x, const V3& org, double h, double* row) {
        double q[3];
        for (int d = 0; d < 3; ++d) q[d] = (x[d] - org[d]) / h + 0.5;
        row[0] = q[0] * q[1] * q[2];
        row[1] = q[0] * q[1];
        row[2] = q[0] * q[2];
        row[3] = q[1] * q[2];
        row[4] = q[0];
        row[5] = q[1];
        row[6] = q[2];
        row[7] = 1.0;
    }
    static void vdmBoundary(const V3& x, const V3& n, const V3& org, double h, double* row) {
        double q[3];
        for (int d = 0; d < 3; ++d) q[d] = (x[d] - org[d]) / h + 0.5;
        row[0] = n[0] * q[1] * q[2] + n[1] * q[0] * q[2] + n[2] * q[0] * q[1];
        row[1] = n[0] * q[1] + n[1] * q[0];
        row[2] = n[0] * q[2] + n[2] * q[0];
        row[3] = n[1] * q[2] + n[2] * q[1];
        row[4] = n[0];
        row[5] = n[1];
        row[6] = n[2];
        row[7] = 0.0;
    }
    // Condition number of the 8 x 8 matrix M from the eigenvalues of M^T M (cyclic
    // Jacobi), and the solution of M w = v (Gaussian elimination with partial
    // pivoting; a singular M gets the minimum-norm least-squares solution from the
    // same eigen-decomposition).
    static double conditionAndSolve(const double M[8][8], const double v[8], double w[8]) {
        double G[8][8], Q[8][8];
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) {
                double a = 0.0;
                for (int k = 0; k < 8; ++k) a += M[k][i] * M[k][j];
                G[i][j] = a;
                Q[i][j] = (i == j) ? 1.0 : 0.0;
            }
        for (int sweep = 0; sweep < 100; ++sweep) {
            double off = 0.0;
            for (int i = 0; i < 8; ++i)
                for (int j = i + 1; j < 8; ++j) off += G[i][j] * G[i][j];
            if (off < 1e-300) break;
            for (int p = 0; p < 8; ++p)
                for (int q = p + 1; q < 8; ++q) {
                    if (std::fabs(G[p][q]) < 1e-300) continue;
                    const double th = (G[q][q] - G[p][p]) / (2.0 * G[p][q]);
                    const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                    const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                    for (int k = 0; k < 8; ++k) {
                        const double gp = G[k][p], gq = G[k][q];
                        G[k][p] = c * gp - sn * gq;
                        G[k][q] = sn * gp + c * gq;
                    }
                    for (int k = 0; k < 8; ++k) {
                        const double gp = G[p][k], gq = G[q][k];
                        G[p][k] = c * gp - sn * gq;
                        G[q][k] = sn * gp + c * gq;
                    }
                    for (int k = 0; k < 8; ++k) {
                        const double qp = Q[k][p], qq = Q[k][q];
                        Q[k][p] = c * qp - sn * qq;
                        Q[k][q] = sn * qp + c * qq;
                    }
                }
        }
        double lmax = 0.0, lmin = 1e300;
        for (int i = 0; i < 8; ++i) {
            lmax = std::max(lmax, G[i][i]);
            lmin = std::min(lmin, G[i][i]);
        }
        const double smax = std::sqrt(std::max(lmax, 0.0)), smin = std::sqrt(std::max(lmin, 0.0));
        const double thr = 8.0 * 2.220446049250313e-16 * smax;
        if (smin > thr) {
            double A[8][9];
            for (int i = 0; i < 8; ++i) {
                for (int j = 0; j < 8; ++j) A[i][j] = M[i][j];
                A[i][8] = v[i];
            }
            for (int c = 0; c < 8; ++c) {
                int piv = c;
                for (int r = c + 1; r < 8; ++r)
                    if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
                for (int j = 0; j < 9; ++j) std::swap(A[c][j], A[piv][j]);
                for (int r = c + 1; r < 8; ++r) {
                    const double f = A[r][c] / A[c][c];
                    for (int j = c; j < 9; ++j) A[r][j] -= f * A[c][j];
                }
            }
            for (int i = 7; i >= 0; --i) {
                double a = A[i][8];
                for (int j = i + 1; j < 8; ++j) a -= A[i][j] * w[j];
                w[i] = a / A[i][i];
            }
        } else {
            // w = Q diag(1/lambda) Q^T M^T v over the eigenvalues above the threshold
            double mtv[8], y[8];
            for (int i = 0; i < 8; ++i) {
                double a = 0.0;
                for (int k = 0; k < 8; ++k) a += M[k][i] * v[k];
                mtv[i] = a;
            }
            for (int j = 0; j < 8; ++j) {
                double a = 0.0;
                for (int i = 0; i < 8; ++i) a += Q[i][j] * mtv[i];
                y[j] = std::sqrt(std::max(G[j][j], 0.0)) > thr ? a / G[j][j] : 0.0;
            }
            for (int i = 0; i < 8; ++i) {
                double a = 0.0;
                for (int j = 0; j < 8; ++j) a += Q[i][j] * y[j];
                w[i] = a;
            }
        }
        return smin > 0.0 ? smax / smin : std::numeric_limits<double>::infinity();
    }

    void PML_pressureUpdateGhostCells_FullyCoupled(const std::vector<double>& p, double t) {
        const int n = (int)ghosts.size();
        if (n == 0) return;
        std::vector<Key> keys;
        keys.reserve(n);
        for (auto& m : ghosts) keys.push_back(m.first);
        std::map<Key, int> rowOf;
        for (int i = 0; i < n; ++i) rowOf[keys[i]] = i;
        std::vector<double> diag(n, 1.0), rhs(n, 0.0);
        std::vector<std::vector<std::pair<int, double>>> off(n);
        for (int r = 0; r < n; ++r) {
            const GhostCell& gc = ghosts.at(keys[r]);
            const double p_neig = p[gc.neighbour];
            if (gc.type == 1) {  // plane constraint: perfectly reflecting
                rhs[r] = p_neig;
                continue;
            }
            const Obj& o = objs[gc.boundaryObject];
            V3 image, bp, ne;
            double dist = gc.distance;
            o.Reflect(gc.position, image, bp, ne, dist);
            const V3 a = o.accel(bp, t);
            V3 g;
            for (int d = 0; d < 3; ++d) g[d] = a[d] * (-rho);
            V3 ncell;
            ncell[std::abs(gc.topology) - 1] = gc.topology > 0 ? 1.0 : -1.0;
            const double g_nr = g[0] * ncell[0] + g[1] * ncell[1] + g[2] * ncell[2];
            const double g_ne = g[0] * ne[0] + g[1] * ne[1] + g[2] * ne[2];
            const double pg = p_neig - 0.75 * h * g_nr;
            const double fdw = o.DistanceToMesh(gc.position) < DISTANCE_TOLERANCE ? -2.0 * std::fabs(dist) : -std::fabs(dist);
            double weighted = g_ne * fdw;
            std::vector<int> nb;
            enclosingNeighbours(image, nb);
            if (nb.size() != 8) {
                rhs[r] = pg;
                continue;
            }
            V3 org;
            for (int q = 0; q < 8; ++q) {
                const V3 cp = cellPosition(nb[q]);
                for (int d = 0; d < 3; ++d) org[d] += cp[d];
            }
            for (int d = 0; d < 3; ++d) org[d] /= 8.0;
            double Vr[8][8], vrow[8], rv[8] = {0};
            int si = -1;
            std::set<int> known;
            std::map<int, Key> unknown;
            vdmRegular(image, org, h, vrow);
            for (int q = 0; q < 8; ++q) {
                const int ci = nb[q];
                if (ci == gc.owner) {
                    vdmBoundary(bp, ne, org, h, Vr[q]);
                    rv[q] = g_ne * h;
                    si = q;
                } else if (!isGhost[ci]) {
                    vdmRegular(cellPosition(ci), org, h, Vr[q]);
                    rv[q] = p[ci];
                    known.insert(q);
                } else {
                    double best = std::numeric_limits<double>::max();
                    Key bestKey = 0;
                    for (const Key kk : ghostTree.at(ci)) {
                        const GhostCell& gn = ghosts.at(kk);
                        double d2 = 0.0;
                        for (int d = 0; d < 3; ++d) d2 += (gn.position[d] - image[d]) * (gn.position[d] - image[d]);
                        if (d2 < best) {
                            best = d2;
                            bestKey = kk;
                        }
                    }
                    vdmRegular(ghosts.at(bestKey).position, org, h, Vr[q]);
                    unknown[q] = bestKey;
                }
            }
            // V^T w = v^T
            double M[8][8], w[8];
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) M[i][j] = Vr[j][i];
            const double cond = conditionAndSolve(M, vrow, w);
            if (cond > CONDN_LIM && si != -1) {
                for (int q = 0; q < 8; ++q) w[q] = rv[q] = 0.0;
                known.clear();
                unknown.clear();
                weighted = pg;
            }
            diag[r] = -1.0;
            double b = -weighted;
            for (const int q : known) b -= w[q] * rv[q];
            if (si != -1) b -= w[si] * rv[si];
            for (const auto& m : unknown) off[r].push_back({rowOf.at(m.second), w[m.first]});
            rhs[r] = b;
        }
        // BiCGSTAB with the diagonal preconditioner, tolerance eps relative to |b|
        auto apply = [&](const std::vector<double>& x, std::vector<double>& y) {
            for (int r = 0; r < n; ++r) {
                double a = diag[r] * x[r];
                for (const auto& e : off[r]) a += e.second * x[e.first];
                y[r] = a;
            }
        };
        auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += a[i] * b[i];
            return s;
        };
        std::vector<double> x(n, 0.0), rr = rhs, r0 = rhs, pv(n, 0.0), v(n, 0.0), y(n), sv(n), z(n), tv(n), ax(n);
        const double eps = 2.220446049250313e-16;
        const double rhs2 = dot(rhs, rhs);
        int it = 0;
        if (rhs2 > 0.0) {
            const double tol2 = eps * eps * rhs2;
            double r0sq = rhs2, rho = 1.0, alpha = 1.0, om = 1.0, res = rhs2;
            int restarts = 0;
            const int maxit = std::min(2 * n, 1000);
            while (res > tol2 && it < maxit) {
                const double rhoOld = rho;
                rho = dot(r0, rr);
                if (std::fabs(rho) < eps * eps * r0sq) {
                    apply(x, ax);
                    for (int i = 0; i < n; ++i) rr[i] = rhs[i] - ax[i];
                    r0 = rr;
                    rho = r0sq = dot(rr, rr);
                    if (restarts++ == 0) it = 0;
                }
                const double beta = (rho / rhoOld) * (alpha / om);
                for (int i = 0; i < n; ++i) pv[i] = rr[i] + beta * (pv[i] - om * v[i]);
                for (int i = 0; i < n; ++i) y[i] = pv[i] / diag[i];
                apply(y, v);
                alpha = rho / dot(r0, v);
                for (int i = 0; i < n; ++i) sv[i] = rr[i] - alpha * v[i];
                for (int i = 0; i < n; ++i) z[i] = sv[i] / diag[i];
                apply(z, tv);
                const double tt = dot(tv, tv);
                om = tt > 0.0 ? dot(tv, sv) / tt : 0.0;
                for (int i = 0; i < n; ++i) {
                    x[i] += alpha * y[i] + om * z[i];
                    rr[i] = sv[i] - om * tv[i];
                }
                res = dot(rr, rr);
                ++it;
            }
        }
        fcIterations = it;
        for (int r = 0; r < n; ++r) ghosts.at(keys[r]).pressure = x[r];
    }

    // MAC_Grid::PML_velocityUpdateCollocated (MAC_Grid.cpp:461-479)
    void PML_velocityUpdateCollocated(const std::vector<double>& pFull) {
#pragma omp parallel for schedule(static)
        for (long ii = 0; ii < (long)pmlV.size(); ++ii) {
            const PMLVCell& cell = pmlV[ii];
            double& v = vel[cell.dim][cell.index];
            v *= cell.upd;
            v += cell.grad * pFull[cell.pr];
            v -= cell.grad * pFull[cell.pl];
        }
    }

    double ghostPressure(int owner, int nbr) const { return ghosts.at(MakeKey(nbr, owner)).pressure; }

    // MAC_Grid::pressureFieldLaplacianGhostCell, default branch (MAC_Grid.cpp:187-299)
    void pressureFieldLaplacianGhostCell(const std::vector<double>& value, std::vector<double>& L) {
        const double scale = 1.0 / (h * h);
        std::fill(L.begin(), L.end(), 0.0);
#pragma omp parallel for schedule(static)
        for (int ci = 0; ci < ncell; ++ci) {
            if (!isBulk[ci]) continue;
            int surroundedDims = 0;
            int ijk[3];
            cellIJK(ci, ijk);
            for (int dim = 0; dim < 3; ++dim) {
                int bp[3] = {ijk[0], ijk[1], ijk[2]}, bn[3] = {ijk[0], ijk[1], ijk[2]};
                if (ijk[dim] != N[dim] - 1) bp[dim] += 1;
                if (ijk[dim] != 0) bn[dim] -= 1;
                const int iP = cellIndex(bp[0], bp[1], bp[2]);
                const int iN = cellIndex(bn[0], bn[1], bn[2]);
                const bool gP = isGhost[iP], gN = isGhost[iN];
                if (gP && gN) {
                    L[ci] += (ghostPressure(iP, ci) + ghostPressure(iN, ci) - 2.0 * value[ci]) / (9.0 / 16.0);
                    ++surroundedDims;
                } else if (gP && !gN) {
                    L[ci] += (ghostPressure(iP, ci) + 0.75 * value[iN] - (7.0 / 4.0) * value[ci]) / (21.0 / 32.0);
                } else if (!gP && gN) {
                    L[ci] += (0.75 * value[iP] + ghostPressure(iN, ci) - (7.0 / 4.0) * value[ci]) / (21.0 / 32.0);
                } else {
                    L[ci] += (value[iP] + value[iN] - 2.0 * value[ci]);
                }
            }
            isCavity[ci] = (surroundedDims > 1);
            L[ci] *= scale;
        }
    }

    // A neighbour's pressure as the Engquist branch reads it: the ghost
    // pressure of the face (ci, nb) when nb is a ghost cell, else buf[nb].
    double engquistValue(int ci, int nb, const std::vector<double>& buf) {
        if (!isGhost[nb]) return buf[nb];
        const auto it = ghosts.find(MakeKey(nb, ci));
        if (it == ghosts.end()) {
            engquistMissingGhost = true;  // the reference's map lookup throws here
            return 0.0;
        }
        return it->second.pressure;
    }

    // The Engquist-Majda absorbing update of a non-PML bulk cell one cell from
    // the domain edge (MAC_Grid.cpp:533-920, ENGQUIST_ORDER 2 for faces; the
    // edge and corner forms the reference keeps are first order).  nml: the
    // cell's boundary normal at offset 1.  Writes the extrapolated exterior
    // pressures into pCurr (zero at the diagonal exterior cell), as the
    // reference does, and returns pNext before the source term.  No boundary
    // interface exists in a single solve, so every blend is the ABC value.
    double engquistUpdate(int ci, const int ijk[3], const int nml[3], const std::vector<double>& pLast,
                          std::vector<double>& pCurr) {
        const double lambda = c * k / h;
        const double lambda2 = lambda * lambda;
        const int btype = std::abs(nml[0]) + std::abs(nml[1]) + std::abs(nml[2]);
        const double pC = pCurr[ci], pL = pLast[ci];
        if (btype == 1) {
            int di = 0;
            while (nml[di] == 0) ++di;
            const int dj = (di + 1) % 3, dk = (di + 2) % 3;
            const int ii = ijk[di], jj = ijk[dj], kk = ijk[dk];
            const int ii_n = ii - nml[di], ii_p = ii + nml[di];
            const int jj_n = std::max(jj - 1, 0), jj_p = std::min(jj + 1, N[dj] - 1);
            const int kk_n = std::max(kk - 1, 0), kk_p = std::min(kk + 1, N[dk] - 1);
            const int nIp = cellIndexP(di, dj, dk, ii_p, jj, kk), nIn = cellIndexP(di, dj, dk, ii_n, jj, kk);
            const int nJp = cellIndexP(di, dj, dk, ii, jj_p, kk), nJn = cellIndexP(di, dj, dk, ii, jj_n, kk);
            const int nKp = cellIndexP(di, dj, dk, ii, jj, kk_p), nKn = cellIndexP(di, dj, dk, ii, jj, kk_n);
            const double pl_ii_p = engquistValue(ci, nIp, pLast);
            const double p_ii_n = engquistValue(ci, nIn, pCurr), pl_ii_n = engquistValue(ci, nIn, pLast);
            const double p_jj_p = engquistValue(ci, nJp, pCurr);
            const double p_jj_n = engquistValue(ci, nJn, pCurr);
            const double p_kk_p = engquistValue(ci, nKp, pCurr);
            const double p_kk_n = engquistValue(ci, nKn, pCurr);
            double p1 = (2. / lambda2 + 4. / lambda - 6. - 4. * lambda) * pC - (1. / lambda2 + 2. / lambda) * pL +
                        pl_ii_p - pl_ii_n + 2. * p_ii_n + (lambda + 1.) * (p_jj_p + p_jj_n + p_kk_p + p_kk_n);
            p1 *= (lambda2 / (1. + 2. * lambda));
            double p_ii_p;
            if (isGhost[nIp]) {
                p_ii_p = engquistValue(ci, nIp, pCurr);
            } else {
                p_ii_p = pl_ii_p + p_ii_n - pl_ii_n - 2. / lambda * (p1 + pL - 2. * pC) +
                         lambda * (p_jj_p + p_jj_n + p_kk_p + p_kk_n - 4. * pC);
            }
            pCurr[nIp] = p_ii_p;
            return 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_p + p_jj_n + p_kk_p + p_kk_n + p_ii_p - 6. * pC);
        }
        if (btype == 2) {
            int di = 0;
            while (nml[di] == 0) ++di;
            int dj = di + 1;
            while (nml[dj] == 0) ++dj;
            const int dk = dj != di + 1 ? (di + 1) % 3 : (di + 2) % 3;
            const int ii = ijk[di], jj = ijk[dj], kk = ijk[dk];
            const int ii_n = ii - nml[di], jj_n = jj - nml[dj];
            const int ii_p = ii + nml[di], jj_p = jj + nml[dj];
            const int kk_n = std::max(kk - 1, 0), kk_p = std::min(kk + 1, N[dk] - 1);
            const double p_ii_n = engquistValue(ci, cellIndexP(di, dj, dk, ii_n, jj, kk), pCurr);
            const double p_jj_n = engquistValue(ci, cellIndexP(di, dj, dk, ii, jj_n, kk), pCurr);
            const double p_kk_p = engquistValue(ci, cellIndexP(di, dj, dk, ii, jj, kk_p), pCurr);
            const double p_kk_n = engquistValue(ci, cellIndexP(di, dj, dk, ii, jj, kk_n), pCurr);
            double p1 = (2. / lambda2 - 6.) * pC + (2.0 * lambda - 1.0) / lambda2 * pL + 2. * p_ii_n + 2. * p_jj_n +
                        p_kk_p + p_kk_n;
            p1 *= (lambda2 / (1. + 2. * lambda));
            const int nIp = cellIndexP(di, dj, dk, ii_p, jj, kk), nJp = cellIndexP(di, dj, dk, ii, jj_p, kk);
            const double p_ii_p = isGhost[nIp] ? engquistValue(ci, nIp, pCurr) : (pL - p1) / lambda + p_ii_n;
            const double p_jj_p = isGhost[nJp] ? engquistValue(ci, nJp, pCurr) : (pL - p1) / lambda + p_jj_n;
            pCurr[nIp] = p_ii_p;
            pCurr[nJp] = p_jj_p;
            pCurr[cellIndexP(di, dj, dk, ii_p, jj_p, kk)] = 0.0;
            return 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_n + p_kk_p + p_kk_n + p_ii_p + p_jj_p - 6. * pC);
        }
        // corner
        const int ii = ijk[0], jj = ijk[1], kk = ijk[2];
        const int ii_n = ii - nml[0], jj_n = jj - nml[1], kk_n = kk - nml[2];
        const int ii_p = ii + nml[0], jj_p = jj + nml[1], kk_p = kk + nml[2];
        const double p_ii_n = engquistValue(ci, cellIndex(ii_n, jj, kk), pCurr);
        const double p_jj_n = engquistValue(ci, cellIndex(ii, jj_n, kk), pCurr);
        const double p_kk_n = engquistValue(ci, cellIndex(ii, jj, kk_n), pCurr);
        double p1 = (2. / lambda2 - 6.) * pC + (3.0 * lambda - 1.0) / lambda2 * pL + 2. * p_ii_n + 2. * p_jj_n +
                    2. * p_kk_n;
        p1 *= (lambda2 / (1. + 3. * lambda));
        const int nIp = cellIndex(ii_p, jj, kk), nJp = cellIndex(ii, jj_p, kk), nKp = cellIndex(ii, jj, kk_p);
        const double p_ii_p = isGhost[nIp] ? engquistValue(ci, nIp, pCurr) : (pL - p1) / lambda + p_ii_n;
        const double p_jj_p = isGhost[nJp] ? engquistValue(ci, nJp, pCurr) : (pL - p1) / lambda + p_jj_n;
        const double p_kk_p = isGhost[nKp] ? engquistValue(ci, nKp, pCurr) : (pL - p1) / lambda + p_kk_n;
        pCurr[nIp] = p_ii_p;
        pCurr[nJp] = p_jj_p;
        pCurr[nKp] = p_kk_p;
        pCurr[cellIndex(ii_p, jj_p, kk_p)] = 0.0;
        return 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_n + p_kk_n + p_ii_p + p_jj_p + p_kk_p - 6. * pC);
    }

    // MAC_Grid::PML_pressureUpdateCollocated (MAC_Grid.cpp:481-946).  Non-PML
    // bulk cells on the domain edge are left as they are; those one cell inside
    // it take the Engquist-Majda update (live only where a side has no PML:
    // presets 1 / 2, or a PML under 1.5 cells).
    void PML_pressureUpdateCollocated(double t, std::vector<double>& pLast, std::vector<double>& pCurr,
                                      std::vector<double>& pNext, const std::vector<double>& lapC,
                                      const std::vector<double>& lapL) {
        const double one_over_dx = 1.0 / h;
        const double c2_k2 = (c * k) * (c * k);
        const double kcalp = c * alpha * k;
        const bool evalSrc = !srcs.empty();
        // PML cells (serial in the reference, independent per cell)
#pragma omp parallel for schedule(static)
        for (long ii = 0; ii < (long)pmlP.size(); ++ii) {
            const PMLPCell& cell = pmlP[ii];
            const int ci = cell.index;
            for (int dim = 0; dim < 3; ++dim) {
                double& pd = pDir[dim][ci];
                pd *= cell.upd[dim];
                pd += cell.div[dim] * vel[dim][cell.vr[dim]] * one_over_dx;
                pd -= cell.div[dim] * vel[dim][cell.vl[dim]] * one_over_dx;
            }
            pNext[ci] = pDir[0][ci] + pDir[1][ci] + pDir[2][ci];
        }
#pragma omp parallel for schedule(static)
        for (int ci = 0; ci < ncell; ++ci) {
            if (!isBulk[ci] || isPML[ci]) continue;
            const V3 pos = cellPosition(ci);
            int ijk[3], nml[3], nml0[3];
            cellIJK(ci, ijk);
            boundaryCellNormal(ijk, 1, nml);
            boundaryCellNormal(ijk, 0, nml0);
            if (nml0[0] != 0 || nml0[1] != 0 || nml0[2] != 0) continue;
            if (nml[0] != 0 || nml[1] != 0 || nml[2] != 0) {
                pNext[ci] = engquistUpdate(ci, ijk, nml, pLast, pCurr);
            } else if (isCavity[ci] && validHistory[ci]) {
                pNext[ci] = pLast[ci] = pCurr[ci];
            } else if (alpha > 0.0 && validHistory[ci]) {
                pNext[ci] = 2.0 * pCurr[ci] - pLast[ci] - lapL[ci] * kcalp + lapC[ci] * (c2_k2 + kcalp);
            } else {
                pNext[ci] = 2.0 * pCurr[ci] - pLast[ci] + lapC[ci] * c2_k2;
            }
            if (evalSrc) pNext[ci] += EvaluatePressureSources(pos, t + 0.5 * k) * k;
        }
    }

    // MLSModeInterpolator::lookup, order 1, Fleishman weights
    // (MLSModeInterpolator.hpp:282-431, :588-598).  The weighted least-squares
    // minimiser is computed by Householder QR; the reference's JacobiSVD
    // returns the same minimiser for a full-rank stencil.
    static bool mls_c0(const V3& p, const std::vector<V3>& pts, const std::vector<double>& val, double& out) {
        const int n = (int)pts.size();
        const double r2 = MLS_FLEISHMAN_RAD * MLS_FLEISHMAN_RAD;
        std::vector<double> A((size_t)n * 4), b(n);
        for (int i = 0; i < n; ++i) {
            const double dx = pts[i][0] - p[0], dy = pts[i][1] - p[1], dz = pts[i][2] - p[2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            const double w = std::exp(-(d2) / (2. * r2));
            A[i * 4 + 0] = 1.0 * w;
            A[i * 4 + 1] = dx * w;
            A[i * 4 + 2] = dy * w;
            A[i * 4 + 3] = dz * w;
            b[i] = val[i] * w;
        }
        return householder_ls4(A.data(), b.data(), n, out);
    }

   public:
    // Householder QR least squares on an n x 4 row-major matrix; returns c[0].
    static bool householder_ls4(double* A, double* b, int n, double& c0) {
        double R[4][4] = {{0}};
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int i = j; i < n; ++i) s += A[i * 4 + j] * A[i * 4 + j];
            const double norm = std::sqrt(s);
            if (!(norm > 0.0)) return false;
            const double x0 = A[j * 4 + j];
            const double alpha_ = x0 > 0.0 ? -norm : norm;
            // v = x - alpha e1, stored in A[j.., j]
            A[j * 4 + j] = x0 - alpha_;
            double vnorm2 = 0.0;
            for (int i = j; i < n; ++i) vnorm2 += A[i * 4 + j] * A[i * 4 + j];
            // apply H = I - 2 v v^T / (v^T v) to remaining columns and b
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
            R[j][j] = alpha_;
            for (int cc = j + 1; cc < 4; ++cc) R[j][cc] = A[j * 4 + cc];
        }
        const double rmax = std::max(std::max(std::fabs(R[0][0]), std::fabs(R[1][1])),
                                     std::max(std::fabs(R[2][2]), std::fabs(R[3][3])));
        for (int j = 0; j < 4; ++j)
            if (std::fabs(R[j][j]) <= (double)std::max(n, 4) * 2.220446049250313e-16 * rmax) return false;
        double x[4];
        for (int j = 3; j >= 0; --j) {
            double s = b[j];
            for (int cc = j + 1; cc < 4; ++cc) s -= R[j][cc] * x[cc];
            x[j] = s / R[j][j];
        }
        c0 = x[0];
        return true;
    }

    // ScalarField::enclosingNeighbours (ScalarField.cpp:261-286), ascending flat index
    void enclosingNeighbours(const V3& x, std::vector<int>& out) const {
        V3 diff;
        for (int d = 0; d < 3; ++d) diff[d] = x[d] - bmin[d];
        for (int d = 0; d < 3; ++d) diff[d] -= h / 2.0;
        int a0[3], a1[3];
        for (int d = 0; d < 3; ++d) {
            a0[d] = std::min(std::max((int)(diff[d] / h), 0), N[d] - 1);
            a1[d] = (diff[d] < 0.0 ? 0 : std::min(a0[d] + 1, N[d] - 1));
        }
        std::set<int> s;
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int l = 0; l < 2; ++l)
                    s.insert(cellIndex(i ? a1[0] : a0[0], j ? a1[1] : a0[1], l ? a1[2] : a0[2]));
        out.assign(s.begin(), s.end());
    }

    // PML_WaveSolver::FetchScalarData (PML_WaveSolver.cpp:210-317)
    int FetchScalarData(const std::vector<double>& scalar, double* data) {
        const int L = (int)listeners.size();
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
        for (int li = 0; li < L; ++li) {
            const V3& point = listeners[li];
            std::vector<int> nb;
            enclosingNeighbours(point, nb);
            std::vector<V3> pts;
            std::vector<double> vals;
            std::vector<int> kept;
            for (int cell : nb) {
                if (std::isnan(scalar[cell])) continue;
                kept.push_back(cell);
                if (!isGhost[cell]) {
                    pts.push_back(cellPosition(cell));
                    vals.push_back(scalar[cell]);
                } else {
                    for (Key key : ghostTree.at(cell)) {
                        const GhostCell& gc = ghosts.at(key);
                        pts.push_back(gc.position);
                        vals.push_back(gc.pressure);
                    }
                }
            }
            if (kept.empty()) { bad++; data[li] = 0.0; continue; }
            if (kept.size() < 4) {
                int best = -1;
                double bestD = DMAX;
                for (int cell : kept) {
                    const V3 cp = cellPosition(cell);
                    const double dx = cp[0] - point[0], dy = cp[1] - point[1], dz = cp[2] - point[2];
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 < bestD) { best = cell; bestD = d2; }
                }
                data[li] = scalar[best];
            } else {
                double c0 = 0.0;
                if (!mls_c0(point, pts, vals, c0)) { bad++; c0 = 0.0; }
                data[li] = c0;
            }
        }
        return bad;
    }

    // PML_WaveSolver::Reinitialize_PML_WaveSolver (PML_WaveSolver.cpp:102-146) followed by
    // FDTD_AcousticSimulator::ResetStartTime (FDTD_AcousticSimulator.cpp:458-523).
    void Reinitialize(double startTime) {
        currentTime = startTime;
        stateTime = startTime;
        timeIndex = 0;
        for (int i = 0; i < 3; ++i) {
            std::fill(pCol[i].begin(), pCol[i].end(), 0.0);
            std::fill(pDir[i].begin(), pDir[i].end(), 0.0);
            std::fill(vel[i].begin(), vel[i].end(), 0.0);
        }
        std::fill(lap[0].begin(), lap[0].end(), 0.0);
        std::fill(lap[1].begin(), lap[1].end(), 0.0);
        pColInd = 1;
        lapInd = 1;
        for (auto& o : objs) { o.pose(startTime); o.UpdateBoundingBox(); o.ResetUnionBox(); }
        // initFieldRasterized -> classifyCells: no boundary fields, every cell bulk
        std::fill(isBulk.begin(), isBulk.end(), 1);
        std::fill(isGhost.begin(), isGhost.end(), 0);
        std::fill(validHistory.begin(), validHistory.end(), 1);  // ResetCellHistory(true)
        classifyCells_FAST();
        std::fill(validHistory.begin(), validHistory.end(), 1);  // ResetCellHistory(true)
    }

    // MAC_Grid::InterpolateFreshPressureCell, MLS branch (MAC_Grid.cpp:1993-2254)
    int InterpolateFreshPressureCell(std::vector<double>& p, double t) {
        for (int ci = 0; ci < ncell; ++ci) {
            if (validHistory[ci] || !isBulk[ci]) continue;
            const V3 cp = cellPosition(ci);
            double distance = DMAX;
            int oid = 0;
            LowestObjectDistance(cp, distance, oid);
            if (distance < DISTANCE_TOLERANCE) { err = "fresh cell inside object"; return FDTD_ERR_GEOMETRY; }
            const Obj& o = objs[oid];
            V3 image, bp, nrm;
            double travelled;
            o.Reflect(cp, image, bp, nrm, travelled);
            std::vector<int> nb;
            enclosingNeighbours(image, nb);
            std::vector<int> kept;
            std::vector<V3> pts;
            std::vector<double> vals;
            for (int n : nb) {
                if (!validHistory[n]) continue;
                kept.push_back(n);
                pts.push_back(cellPosition(n));
                vals.push_back(p[n]);
            }
            if (kept.size() < 4) {
                if (!kept.empty()) {
                    double md = DMAX;
                    int mid = -1;
                    for (int n : kept) {
                        const V3 q = cellPosition(n);
                        const double dx = image[0] - q[0], dy = image[1] - q[1], dz = image[2] - q[2];
                        const double d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 < md) { md = d2; mid = n; }
                    }
                    p[ci] = p[mid];
                } else {
                    int ijk[3];
                    cellIJK(ci, ijk);
                    int best = -1;
                    for (int dim = 0; dim < 3 && best < 0; ++dim) {
                        for (int s = 1; s >= -1 && best < 0; s -= 2) {
                            int a[3] = {ijk[0], ijk[1], ijk[2]};
                            a[dim] += s;
                            if (a[dim] < 0 || a[dim] >= N[dim]) continue;
                            const int ii = cellIndex(a[0], a[1], a[2]);
                            if (isBulk[ii]) best = ii;
                        }
                    }
                    p[ci] = best >= 0 ? p[best] : 0.0;
                }
            } else {
                double c0 = 0.0;
                if (!mls_c0(image, pts, vals, c0)) c0 = 0.0;
                const V3 acc = o.accel(bp, t);
                const double an = acc[0] * nrm[0] + acc[1] * nrm[1] + acc[2] * nrm[2];
                p[ci] = c0 + rho * an * std::fabs(travelled);
            }
        }
        return FDTD_OK;
    }

    // PML_WaveSolver::stepCollocated, non-FV branch (PML_WaveSolver.cpp:775-826)
    // followed by the listener fetch and object update of SimWorld::StepWorld
    // (SimWorld.cpp:507-600).
    int step(double* listener_row) {
        std::vector<double>& pLast = pCol[(pColInd + 2) % 3];
        std::vector<double>& pCurr = pCol[pColInd];
        std::vector<double>& pNext = pCol[(pColInd + 1) % 3];
        std::vector<double>& lapLast = lap[(lapInd + 1) % 2];
        std::vector<double>& lapCurr = lap[lapInd];
        classifyCells_FAST();
        int st = InterpolateFreshPressureCell(pLast, currentTime);
        if (st != FDTD_OK) return st;
        st = InterpolateFreshPressureCell(pCurr, currentTime);
        if (st != FDTD_OK) return st;
        if (fullyCoupled) PML_pressureUpdateGhostCells_FullyCoupled(pCurr, currentTime);
        else PML_pressureUpdateGhostCells(pCurr, currentTime);
        PML_velocityUpdateCollocated(pCurr);
        pressureFieldLaplacianGhostCell(pCurr, lapCurr);
        PML_pressureUpdateCollocated(currentTime, pLast, pCurr, pNext, lapCurr, lapLast);
        if (engquistMissingGhost) {
            err = "an Engquist cell has a ghost neighbour without a face record";
            return FDTD_ERR_UNSUPPORTED;
        }
        pColInd = (pColInd + 1) % 3;
        lapInd = (lapInd + 1) % 2;
        currentTime += k;
        timeIndex += 1;
        int bad = 0;
        if (listener_row) bad = FetchScalarData(pCol[pColInd], listener_row);
        // SimWorld::UpdateObjectState(t + dt) -> animate -> UpdateBoundingBox
        stateTime += k;
        for (auto& o : objs) {
            if (o.d.motion == FDTD_MOTION_STATIC) continue;
            o.pose(stateTime);
            o.UpdateBoundingBox();
        }
        return bad ? FDTD_ERR_NUMERIC : FDTD_OK;
    }

    int init(const fdtd_scene_desc* s) {
        if (!s || s->cell_size <= 0) { err = "bad scene"; return FDTD_ERR_INVALID_ARG; }
        h = s->cell_size;
        c = s->sound_speed;
        rho = s->density;
        k = s->time_step;
        alpha = s->air_viscosity_alpha;
        preset = s->boundary_condition_preset;
        fullyCoupled = s->boundary_handling == FDTD_BOUNDARY_FULLY_COUPLED;
        endTime = s->end_time;
        if (preset < 0 || preset > 2) { err = "boundary_condition_preset must be 0, 1 or 2"; return FDTD_ERR_INVALID_ARG; }
        // BoundingBox(cellSize, divisions, center) (BoundingBox.h:89-99), per-axis divisions
        V3 mn, mx;
        for (int d = 0; d < 3; ++d) {
            mn[d] = s->domain_center[d] - h * (double)s->divisions[d] / 2.0;
            mx[d] = s->domain_center[d] + h * (double)s->divisions[d] / 2.0;
        }
        // ScalarField(bbox, cellSize) (ScalarField.cpp:29-50)
        for (int d = 0; d < 3; ++d) {
            N[d] = (int)std::ceil(((mx[d] - mn[d]) - EPS) / h);
            bmin[d] = mn[d];
            bmax[d] = bmin[d];
            bmax[d] += h * (double)N[d];
        }
        ncell = N[0] * N[1] * N[2];
        // MAC_Grid::Reinitialize_MAC_Grid (MAC_Grid.cpp:90-134)
        for (int dim = 0; dim < 3; ++dim) {
            for (int d = 0; d < 3; ++d) { vN[dim][d] = N[d] + (d == dim ? 1 : 0); vmin[dim][d] = bmin[d]; }
            vmin[dim][dim] = bmin[dim] - h / 2.0;
        }
        absorptionWidth = s->pml_width * h;  // setPMLBoundaryWidth (MAC_Grid.cpp:146-150)
        absorptionStrength = s->pml_strength;
        meshes.resize(std::max(0, s->n_meshes));
        for (int m = 0; m < (int)meshes.size(); ++m)
            if (!meshes[m].build(s->meshes[m])) { err = "mesh is open or degenerate"; return FDTD_ERR_GEOMETRY; }
        for (int i = 0; i < s->n_objects; ++i) {
            Obj o;
            o.d = s->objects[i];
            for (int k = 0; k < 9; ++k) o.R0[k] = o.d.rotation[k];
            if (o.d.shape == FDTD_SHAPE_MESH) {
                if (o.d.mesh < 0 || o.d.mesh >= (int)meshes.size()) { err = "mesh index"; return FDTD_ERR_INVALID_ARG; }
                o.mesh = &meshes[o.d.mesh];
                o.MeshExtent();
            }
            if (o.d.motion == FDTD_MOTION_KEYFRAMED) {
                for (int k = 0; k < s->n_tracks; ++k)
                    if (s->tracks[k].object == i) {
                        o.kf.assign(s->tracks[k].frames, s->tracks[k].frames + 7 * (size_t)s->tracks[k].n_frames);
                        o.kf_step = s->tracks[k].step;
                    }
                if (o.kf.empty() || !(o.kf_step > 0)) { err = "keyframed object without a track"; return FDTD_ERR_INVALID_ARG; }
            }
            objs.push_back(o);
        }
        for (int i = 0; i < s->n_constraints; ++i) planes.push_back(s->constraints[i]);
        for (int i = 0; i < s->n_sources; ++i) {
            fdtd_gaussian_source_desc g = s->sources[i];
            if (g.width_space <= 0) g.width_space = c * g.width_time;
            if (g.normalize_constant == 0)
                g.normalize_constant = 1.0 / std::pow(std::sqrt(2.0 * M_PI) * g.width_space, 3);
            srcs.push_back(g);
            // GaussianPressureSource ctor bbox (GaussianPressureSource.h:30-37)
            OBox b;
            V3 a, bb;
            for (int d = 0; d < 3; ++d) {
                a[d] = g.position[d] - g.width_space * GAUSSIAN_CHECK_BOUND;
                bb[d] = g.position[d] + g.width_space * GAUSSIAN_CHECK_BOUND;
            }
            b.Update(a, bb);
            srcBox.push_back(b);
        }
        for (int i = 0; i < s->n_listeners; ++i)
            listeners.push_back(V3(s->listeners[3 * i], s->listeners[3 * i + 1], s->listeners[3 * i + 2]));
        for (int i = 0; i < 3; ++i) {
            pCol[i].assign(ncell, 0.0);
            pDir[i].assign(ncell, 0.0);
            vel[i].assign((size_t)vN[i][0] * vN[i][1] * vN[i][2], 0.0);
        }
        lap[0].assign(ncell, 0.0);
        lap[1].assign(ncell, 0.0);
        isBulk.assign(ncell, 1);
        isGhost.assign(ncell, 0);
        isPML.assign(ncell, 0);
        isCavity.assign(ncell, 0);
        validHistory.assign(ncell, 1);
        gcTypeOf.assign(ncell, 0);
        classifyPML();
        Reinitialize(s->start_time);
        return FDTD_OK;
    }
};

}  // namespace

extern "C" {

int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// Signed distance of n points to a mesh in its frame (OMesh::Sdf, every triangle).
int oracle_mesh_sdf(const fdtd_mesh_desc* mesh, long long n, const double* points, double* out) {
    OMesh m;
    if (!mesh || !m.build(*mesh)) return FDTD_ERR_GEOMETRY;
    for (long long i = 0; i < n; ++i) out[i] = m.Sdf(V3(points[3 * i], points[3 * i + 1], points[3 * i + 2]));
    return 0;
}

int oracle_create(const fdtd_scene_desc* scene, void** out) {
    Oracle* o = new Oracle();
    const int st = o->init(scene);
    if (st != FDTD_OK) { delete o; *out = nullptr; return st; }
    *out = o;
    return FDTD_OK;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

int oracle_reset(void* h, double t0) {
    static_cast<Oracle*>(h)->Reinitialize(t0);
    return FDTD_OK;
}

// n steps; listener_out holds n * L doubles (row = step), may be NULL
int oracle_step(void* h, int n, double* listener_out) {
    Oracle* o = static_cast<Oracle*>(h);
    const int L = (int)o->listeners.size();
    std::vector<double> row(L > 0 ? L : 1);
    int result = FDTD_OK;
    for (int i = 0; i < n; ++i) {
        const int st = o->step(listener_out ? row.data() : nullptr);
        if (st == FDTD_ERR_GEOMETRY) return st;
        if (st != FDTD_OK) result = st;
        if (listener_out) std::memcpy(listener_out + (size_t)i * L, row.data(), sizeof(double) * L);
    }
    if (o->endTime > 0.0 && o->currentTime >= o->endTime && result == FDTD_OK) result = FDTD_END_OF_TIME;
    return result;
}

double oracle_time(void* h) { return static_cast<Oracle*>(h)->currentTime; }

int64_t oracle_num_cells(void* h) { return static_cast<Oracle*>(h)->ncell; }
int64_t oracle_num_pml_cells(void* h) { return (int64_t) static_cast<Oracle*>(h)->pmlP.size(); }

int oracle_get_classification(void* h, uint8_t* flags, fdtd_ghost_face* faces, int64_t* n_faces) {
    Oracle* o = static_cast<Oracle*>(h);
    if (flags) {
        for (int i = 0; i < o->ncell; ++i) {
            uint8_t f = 0;
            if (o->isBulk[i]) f |= FDTD_CELL_BULK;
            if (o->isGhost[i]) f |= FDTD_CELL_GHOST;
            if (o->validHistory[i]) f |= FDTD_CELL_VALID_HISTORY;
            if (o->isPML[i]) f |= FDTD_CELL_PML;
            if (!o->isBulk[i] && o->gcTypeOf[i] == 1) f |= FDTD_CELL_CONSTRAINT;
            flags[i] = f;
        }
    }
    // faces ordered by (owner, key)
    std::vector<fdtd_ghost_face> list;
    for (auto& t : o->ghostTree) {
        for (Key key : t.second) {
            const GhostCell& g = o->ghosts.at(key);
            fdtd_ghost_face f;
            std::memset(&f, 0, sizeof(f));
            f.owner_cell = g.owner;
            f.neighbour_cell = g.neighbour;
            f.topology = g.topology;
            f.type = g.type;
            f.boundary_object = g.boundaryObject;
            f.key = key;
            list.push_back(f);
        }
    }
    if (faces) {
        const int64_t cap = *n_faces;
        for (int64_t i = 0; i < (int64_t)list.size() && i < cap; ++i) faces[i] = list[i];
    }
    *n_faces = (int64_t)list.size();
    return FDTD_OK;
}

int oracle_get_field(void* h, int which, double* out, int64_t count) {
    Oracle* o = static_cast<Oracle*>(h);
    const std::vector<double>* src = nullptr;
    switch (which) {
        case FDTD_FIELD_PRESSURE: src = &o->pCol[o->pColInd]; break;
        case FDTD_FIELD_PRESSURE_PREV: src = &o->pCol[(o->pColInd + 2) % 3]; break;
        case FDTD_FIELD_PML_PX: src = &o->pDir[0]; break;
        case FDTD_FIELD_PML_PY: src = &o->pDir[1]; break;
        case FDTD_FIELD_PML_PZ: src = &o->pDir[2]; break;
        case FDTD_FIELD_VX: src = &o->vel[0]; break;
        case FDTD_FIELD_VY: src = &o->vel[1]; break;
        case FDTD_FIELD_VZ: src = &o->vel[2]; break;
        default: return FDTD_ERR_INVALID_ARG;
    }
    if (count != (int64_t)src->size()) return FDTD_ERR_INVALID_ARG;
    std::memcpy(out, src->data(), sizeof(double) * src->size());
    return FDTD_OK;
}

// MAC_Grid::GetCell (MAC_Grid.cpp:4182-4258, non-FV branch) and the stored
// Laplacian of PML_WaveSolver::FetchCell (PML_WaveSolver.cpp:439-447).
int oracle_fetch_cell(void* h, int64_t cell, fdtd_cell* out) {
    Oracle* o = static_cast<Oracle*>(h);
    if (cell < 0 || cell >= o->ncell) return FDTD_ERR_INVALID_ARG;
    const int idx = (int)cell;
    fdtd_cell& c = *out;
    std::memset(&c, 0, sizeof(c));
    c.index = idx;
    int ijk[3];
    o->cellIJK(idx, ijk);
    for (int d = 0; d < 3; ++d) c.indices[d] = ijk[d];
    const V3 pos = o->cellPosition(idx);
    // PressureCellType (MAC_Grid.cpp:3977-3997)
    for (int g = 0; g < 6; ++g) c.gc_value[g] = -1.0;
    if (o->isPML[idx]) {
        double m = std::numeric_limits<double>::min();
        for (int d = 0; d < 3; ++d) m = std::max(m, o->PML_absorptionCoefficient(pos, d));
        c.r_identity = -0.5 * m / o->absorptionStrength;
    } else if (o->isBulk[idx]) {
        c.r_identity = 0.5;
    } else if (!o->isGhost[idx]) {
        c.r_identity = 1.0;
    } else {
        c.r_identity = -1.0;
        c.n_gc_value = 6;
        int count = 0;
        for (int dim = 0; dim < 3; ++dim)
            for (int dir = -1; dir <= 1; dir += 2, ++count) {
                int nb[3] = {ijk[0], ijk[1], ijk[2]};
                nb[dim] += dir;
                if (nb[dim] < 0 || nb[dim] >= o->N[dim]) continue;
                const auto it = o->ghosts.find(MakeKey(idx, o->cellIndex(nb[0], nb[1], nb[2])));
                if (it != o->ghosts.end()) c.gc_value[count] = it->second.pressure;
            }
    }
    uint8_t f = 0;
    if (o->isBulk[idx]) f |= FDTD_CELL_BULK;
    if (o->isGhost[idx]) f |= FDTD_CELL_GHOST;
    if (o->validHistory[idx]) f |= FDTD_CELL_VALID_HISTORY;
    if (o->isPML[idx]) f |= FDTD_CELL_PML;
    if (!o->isBulk[idx] && o->gcTypeOf[idx] == 1) f |= FDTD_CELL_CONSTRAINT;
    c.flags = f | FDTD_CELLINFO_LAPLACIAN | FDTD_CELLINFO_PML_STATE;
    for (int d = 0; d < 3; ++d) {
        c.centroid[d] = pos[d];
        c.lower_corner[d] = pos[d] - o->h / 2.0;
        c.upper_corner[d] = pos[d] + o->h / 2.0;
    }
    for (int d = 0; d < 3; ++d) c.p_directional[d] = o->pDir[d][idx];
    c.p_full = o->pCol[o->pColInd][idx];
    double* vv[3] = {c.vx, c.vy, c.vz};
    for (int d = 0; d < 3; ++d) {
        int up[3] = {ijk[0], ijk[1], ijk[2]};
        up[d] = std::min(up[d] + 1, o->N[d]);
        vv[d][0] = o->vel[d][o->vIndex(d, ijk[0], ijk[1], ijk[2])];
        vv[d][1] = o->vel[d][o->vIndex(d, up[0], up[1], up[2])];
    }
    c.h = o->h;
    c.laplacian = o->lap[o->lapInd][idx];
    return FDTD_OK;
}

// listener values at the current state (FetchPressureData)
int oracle_fetch_listeners(void* h, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    return o->FetchScalarData(o->pCol[o->pColInd], out) ? FDTD_ERR_NUMERIC : FDTD_OK;
}

// weighted least-squares constant term, exported for unit tests of the MLS restatement
int oracle_mls_c0(const double* p, const double* pts, const double* vals, int n, double* out) {
    std::vector<V3> P;
    std::vector<double> v;
    for (int i = 0; i < n; ++i) { P.push_back(V3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2])); v.push_back(vals[i]); }
    double c0 = 0;
    std::vector<double> A((size_t)n * 4), b(n);
    const double r2 = MLS_FLEISHMAN_RAD * MLS_FLEISHMAN_RAD;
    for (int i = 0; i < n; ++i) {
        const double dx = P[i][0] - p[0], dy = P[i][1] - p[1], dz = P[i][2] - p[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double w = std::exp(-(d2) / (2. * r2));
        A[i * 4 + 0] = 1.0 * w;
        A[i * 4 + 1] = dx * w;
        A[i * 4 + 2] = dy * w;
        A[i * 4 + 3] = dz * w;
        b[i] = v[i] * w;
    }
    const bool ok = Oracle::householder_ls4(A.data(), b.data(), n, c0);
    *out = c0;
    return ok ? FDTD_OK : FDTD_ERR_NUMERIC;
}

}  // extern "C"
