// fdtd_mesh.cpp — host side of triangle-mesh bodies: validation of a mesh
// (closed and consistently oriented, as the reference's signed distance field
// requires, AdaptiveDistanceField.cpp:92-96), pseudo-normals of faces, edges
// and vertices [Baerentzen 2002], the bounding-volume hierarchy the device
// queries walk (fdtd_mesh.cuh), and the Wavefront .obj reader
// (MeshObjReader::read with a scale, FDTD_RigidObject.cpp:84-93).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

namespace fdtd {

namespace {

void sub3(const double* a, const double* b, double* r) {
    for (int i = 0; i < 3; ++i) r[i] = a[i] - b[i];
}
void cross3(const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double norm3(const double* a) { return std::sqrt(dot3(a, a)); }

struct Builder {
    const std::vector<MeshTri>* all;
    std::vector<int> order;
    std::vector<MeshNode> nodes;
    int max_depth = 0;

    void bounds(int lo, int hi, double* mn, double* mx) const {
        for (int d = 0; d < 3; ++d) {
            mn[d] = HUGE_VAL;
            mx[d] = -HUGE_VAL;
        }
        for (int k = lo; k < hi; ++k) {
            const MeshTri& t = (*all)[order[k]];
            for (int v = 0; v < 3; ++v)
                for (int d = 0; d < 3; ++d) {
                    mn[d] = std::min(mn[d], t.p[v][d]);
                    mx[d] = std::max(mx[d], t.p[v][d]);
                }
        }
    }

    // node `at` covers order[lo, hi)
    void build(int at, int lo, int hi, int depth) {
        max_depth = std::max(max_depth, depth);
        double mn[3], mx[3];
        bounds(lo, hi, mn, mx);
        // widen the box a little: a triangle's rounded distance is then never below its box's
        double ext = 0.0;
        for (int d = 0; d < 3; ++d) ext = std::max(ext, mx[d] - mn[d]);
        for (int d = 0; d < 3; ++d) {
            const double pad = 1e-9 * (ext + std::max(std::fabs(mn[d]), std::fabs(mx[d])));
            nodes[at].lo[d] = mn[d] - pad;
            nodes[at].hi[d] = mx[d] + pad;
        }
        if (hi - lo <= 4 || depth >= 48) {
            nodes[at].first = lo;
            nodes[at].count = hi - lo;
            return;
        }
        // median split of the centroids along the widest centroid extent
        double cmn[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, cmx[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
        auto centroid = [&](int t, int d) {
            const MeshTri& T = (*all)[t];
            return (T.p[0][d] + T.p[1][d] + T.p[2][d]) / 3.0;
        };
        for (int k = lo; k < hi; ++k)
            for (int d = 0; d < 3; ++d) {
                cmn[d] = std::min(cmn[d], centroid(order[k], d));
                cmx[d] = std::max(cmx[d], centroid(order[k], d));
            }
        int axis = 0;
        for (int d = 1; d < 3; ++d)
            if (cmx[d] - cmn[d] > cmx[axis] - cmn[axis]) axis = d;
        const int mid = (lo + hi) / 2;
        std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi, [&](int a, int b) {
            const double ca = centroid(a, axis), cb = centroid(b, axis);
            return ca < cb || (ca == cb && a < b);
        });
        const int left = (int)nodes.size();
        nodes.resize(nodes.size() + 2);
        nodes[at].first = left;
        nodes[at].count = 0;
        build(left, lo, mid, depth + 1);
        build(left + 1, mid, hi, depth + 1);
    }
};

}  // namespace

bool build_mesh(const fdtd_mesh_desc& md, MeshHost& out, std::string& err) {
    const int nv = md.n_vertices, nt = md.n_triangles;
    if (nv < 4 || nt < 4 || !md.vertices || !md.triangles) {
        err = "mesh: at least 4 vertices and 4 triangles are needed";
        return false;
    }
    for (int i = 0; i < 3 * nv; ++i)
        if (!std::isfinite(md.vertices[i])) {
            err = "mesh: non-finite vertex coordinate";
            return false;
        }
    std::vector<MeshTri> tris(nt);
    std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> edges;  // (a, b) directed -> (tri, local edge)
    for (int t = 0; t < nt; ++t) {
        MeshTri& T = tris[t];
        std::memset(&T, 0, sizeof(T));
        T.id = t;
        int v[3];
        for (int k = 0; k < 3; ++k) {
            v[k] = md.triangles[3 * t + k];
            if (v[k] < 0 || v[k] >= nv) {
                err = "mesh: triangle " + std::to_string(t) + " has a vertex index out of range";
                return false;
            }
            for (int d = 0; d < 3; ++d) T.p[k][d] = md.vertices[3 * v[k] + d];
        }
        if (v[0] == v[1] || v[1] == v[2] || v[0] == v[2]) {
            err = "mesh: triangle " + std::to_string(t) + " repeats a vertex";
            return false;
        }
        double e1[3], e2[3], n[3];
        sub3(T.p[1], T.p[0], e1);
        sub3(T.p[2], T.p[0], e2);
        cross3(e1, e2, n);
        const double ln = norm3(n);
        if (!(ln > 0.0)) {
            err = "mesh: triangle " + std::to_string(t) + " has zero area";
            return false;
        }
        for (int d = 0; d < 3; ++d) T.nf[d] = n[d] / ln;
        for (int k = 0; k < 3; ++k) edges[{v[k], v[(k + 1) % 3]}].push_back({t, k});
    }
    // closed and consistently oriented: each directed edge once, its reverse once
    for (const auto& e : edges) {
        if (e.second.size() != 1) {
            err = "mesh: an edge is used twice in the same direction (inconsistent orientation or non-manifold)";
            return false;
        }
        const auto r = edges.find({e.first.second, e.first.first});
        if (r == edges.end()) {
            err = "mesh has a boundary (an edge with one triangle); a closed surface is required";
            return false;
        }
        const int t = e.second[0].first, k = e.second[0].second, u = r->second[0].first;
        for (int d = 0; d < 3; ++d) tris[t].ne[k][d] = tris[t].nf[d] + tris[u].nf[d];
    }
    // vertices: sum of the incident unit face normals weighted by the incident angle
    std::vector<double> vn(3 * (size_t)nv, 0.0);
    for (int t = 0; t < nt; ++t) {
        for (int k = 0; k < 3; ++k) {
            const double* p = tris[t].p[k];
            double a[3], b[3];
            sub3(tris[t].p[(k + 1) % 3], p, a);
            sub3(tris[t].p[(k + 2) % 3], p, b);
            double c = dot3(a, b) / (norm3(a) * norm3(b));
            c = std::max(-1.0, std::min(1.0, c));
            const double ang = std::acos(c);
            const int v = md.triangles[3 * t + k];
            for (int d = 0; d < 3; ++d) vn[3 * v + d] += ang * tris[t].nf[d];
        }
    }
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k) {
            const int v = md.triangles[3 * t + k];
            for (int d = 0; d < 3; ++d) tris[t].nv[k][d] = vn[3 * v + d];
        }
    // hierarchy
    Builder B;
    B.all = &tris;
    B.order.resize(nt);
    for (int t = 0; t < nt; ++t) B.order[t] = t;
    B.nodes.resize(1);
    B.build(0, 0, nt, 0);
    if (B.max_depth + 2 >= MESH_STACK) {
        err = "mesh: hierarchy too deep";
        return false;
    }
    out.nodes = B.nodes;
    out.tris.resize(nt);
    for (int k = 0; k < nt; ++k) out.tris[k] = tris[B.order[k]];
    out.vertices.assign(md.vertices, md.vertices + 3 * (size_t)nv);
    return true;
}

// Extent of rotation * v over the vertices: the world box of the body is
// centre + [lo, hi] (FDTD_RigidObject::UpdateBoundingBox, FDTD_RigidObject.cpp:190-226).
void mesh_extent(const double* verts, size_t nv, const double R[9], double lo[3], double hi[3]) {
    for (int d = 0; d < 3; ++d) {
        lo[d] = HUGE_VAL;
        hi[d] = -HUGE_VAL;
    }
    for (size_t v = 0; v < nv; ++v) {
        const double* p = &verts[3 * v];
        for (int d = 0; d < 3; ++d) {
            const double w = R[d * 3 + 0] * p[0] + R[d * 3 + 1] * p[1] + R[d * 3 + 2] * p[2];
            lo[d] = std::min(lo[d], w);
            hi[d] = std::max(hi[d], w);
        }
    }
}

bool read_obj(const char* path, double scale, std::vector<double>& verts, std::vector<int32_t>& tris, std::string& err) {
    std::ifstream f(path);
    if (!f) {
        err = std::string("cannot open mesh file ") + path;
        return false;
    }
    verts.clear();
    tris.clear();
    std::string line;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        if (line.size() < 2) continue;
        std::istringstream ss(line);
        std::string tag;
        ss >> tag;
        if (tag == "v") {
            double x, y, z;
            if (!(ss >> x >> y >> z)) {
                err = std::string(path) + ":" + std::to_string(lineno) + ": bad vertex";
                return false;
            }
            verts.push_back(x * scale);
            verts.push_back(y * scale);
            verts.push_back(z * scale);
        } else if (tag == "f") {
            std::vector<int32_t> idx;
            std::string tok;
            while (ss >> tok) {
                // "i", "i/t", "i//n", "i/t/n"; negative indices count from the end
                const long v = std::strtol(tok.c_str(), nullptr, 10);
                const long nvs = (long)(verts.size() / 3);
                const long z = v > 0 ? v - 1 : nvs + v;
                if (v == 0 || z < 0) {
                    err = std::string(path) + ":" + std::to_string(lineno) + ": bad face index";
                    return false;
                }
                idx.push_back((int32_t)z);
            }
            if (idx.size() < 3) {
                err = std::string(path) + ":" + std::to_string(lineno) + ": face with fewer than 3 vertices";
                return false;
            }
            for (size_t k = 1; k + 1 < idx.size(); ++k) {  // fan
                tris.push_back(idx[0]);
                tris.push_back(idx[k]);
                tris.push_back(idx[k + 1]);
            }
        }
    }
    for (int32_t t : tris)
        if (t >= (int32_t)(verts.size() / 3)) {
            err = std::string(path) + ": face index beyond the vertices";
            return false;
        }
    return true;
}

}  // namespace fdtd

extern "C" fdtd_status fdtd_read_obj(const char* path, double scale, int32_t* n_vertices, int32_t* n_triangles,
                                     double* vertices, int32_t* triangles) {
    if (!path || !n_vertices || !n_triangles) return FDTD_ERR_INVALID_ARG;
    std::vector<double> v;
    std::vector<int32_t> t;
    std::string err;
    if (!fdtd::read_obj(path, scale, v, t, err)) {
        fdtd::set_error(nullptr, err);
        return FDTD_ERR_IO;
    }
    *n_vertices = (int32_t)(v.size() / 3);
    *n_triangles = (int32_t)(t.size() / 3);
    if (vertices) std::memcpy(vertices, v.data(), v.size() * sizeof(double));
    if (triangles) std::memcpy(triangles, t.data(), t.size() * sizeof(int32_t));
    return FDTD_OK;
}

extern "C" fdtd_status fdtd_mesh_signed_distance(const fdtd_mesh_desc* mesh, int64_t n, const double* points,
                                                 double* out) {
    if (!mesh || n < 0 || (n > 0 && (!points || !out))) return FDTD_ERR_INVALID_ARG;
    fdtd::MeshHost M;
    std::string err;
    if (!fdtd::build_mesh(*mesh, M, err)) {
        fdtd::set_error(nullptr, err);
        return FDTD_ERR_GEOMETRY;
    }
    const fdtd::MeshView v{M.nodes.data(), M.tris.data(), (int)M.nodes.size(), (int)M.tris.size()};
    for (int64_t i = 0; i < n; ++i) out[i] = fdtd::mesh_sdf(v, points + 3 * i);
    return FDTD_OK;
}
