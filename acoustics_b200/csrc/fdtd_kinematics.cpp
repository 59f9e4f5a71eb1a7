// fdtd_kinematics.cpp — keyframed rigid-body poses (host side).
//
// The reference animates a body from per-frame centre and quaternion:
//   FDTD_RigidObject_Blender_Animator::ReadObjectKinData (FDTD_RigidObject_Animator.cpp:79-122)
//     reads "frame tx ty tz qw qx qy qz" lines, clamps w, turns each rotation by
//     -90 degrees about x (Quaternion::fromAxisRotD, Quaternion.hpp:202-208);
//   GetRigidObjectTransform (FDTD_RigidObject_Animator.cpp:128-155) picks the
//     frames around t, lerps the centre and slerps the rotation
//     (Quaternion::slerp, Quaternion.hpp:392-420);
//   FDTD_Objects::AnimateObjects (FDTD_Objects.cpp:568-580) normalises the
//     quaternion and FDTD_RigidObject::SetRigidBodyTransform
//     (FDTD_RigidObject.cpp:549-566) turns it into an axis-angle rotation about
//     the rest centre followed by the move to the new centre.
// The arithmetic follows those expressions in their order (host code built with
// -ffp-contract=off); the axis-angle matrix is the standard Rodrigues form,
// grouped as Eigen's AngleAxis::toRotationMatrix groups it.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

namespace fdtd {
namespace {

struct Quat {
    double w, x, y, z;
};
constexpr double QUAT_EPS = 1e-12;  // Quaternion<double>::EPS (Quaternion.cpp:29)

double length_sqr(const Quat& q) { return q.w * q.w + (q.x * q.x + q.y * q.y + q.z * q.z); }

void normalize(Quat& q) {
    double len = length_sqr(q);
    if (std::fabs(len - 1.0) > QUAT_EPS) {
        len = 1. / std::sqrt(len);
        q.w *= len;
        q.x *= len;
        q.y *= len;
        q.z *= len;
    }
}

double dot(const Quat& a, const Quat& b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }

Quat mul(const Quat& a, const Quat& b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z, a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x};
}

Quat slerp(const Quat& q0, double r, const Quat& q1) {
    Quat v0 = q0, v1 = q1;
    normalize(v0);
    normalize(v1);
    double d = dot(v0, v1);
    if (std::fabs(d) > 0.9995) {
        Quat ret{v0.w + (v1.w - v0.w) * r, v0.x + (v1.x - v0.x) * r, v0.y + (v1.y - v0.y) * r,
                 v0.z + (v1.z - v0.z) * r};
        normalize(ret);
        return ret;
    }
    if (d < 0.0) {
        v1 = {v1.w * -1.0, v1.x * -1.0, v1.y * -1.0, v1.z * -1.0};
        d = -d;
    }
    d = std::min(std::max(d, -1.0), 1.0);
    const double theta = std::acos(d) * r;
    Quat v2{v1.w - v0.w * d, v1.x - v0.x * d, v1.y - v0.y * d, v1.z - v0.z * d};
    normalize(v2);
    const double c = std::cos(theta), s = std::sin(theta);
    return {v0.w * c + v2.w * s, v0.x * c + v2.x * s, v0.y * c + v2.y * s, v0.z * c + v2.z * s};
}

// SetRigidBodyTransform: toAxisRotR (Quaternion.hpp:298-313), then the axis-angle matrix
void rotation_matrix(const Quat& q, double R[9]) {
    const double angle = 2.0 * std::acos(q.w);
    double a[3] = {0.0, 1.0, 0.0};
    if (!(angle < QUAT_EPS)) {
        a[0] = q.x;
        a[1] = q.y;
        a[2] = q.z;
        const double len = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (len > 0) {
            a[0] /= len;
            a[1] /= len;
            a[2] /= len;
        }
    }
    const double sn = std::sin(angle), cs = std::cos(angle);
    const double sa[3] = {sn * a[0], sn * a[1], sn * a[2]};
    const double ca[3] = {(1.0 - cs) * a[0], (1.0 - cs) * a[1], (1.0 - cs) * a[2]};
    double t = ca[0] * a[1];
    R[0 * 3 + 1] = t - sa[2];
    R[1 * 3 + 0] = t + sa[2];
    t = ca[0] * a[2];
    R[0 * 3 + 2] = t + sa[1];
    R[2 * 3 + 0] = t - sa[1];
    t = ca[1] * a[2];
    R[1 * 3 + 2] = t - sa[0];
    R[2 * 3 + 1] = t + sa[0];
    for (int i = 0; i < 3; ++i) R[i * 3 + i] = ca[i] * a[i] + cs;
}

}  // namespace

void keyframe_pose(const double* frames, int n, double step, double t, double com[3], double R[9]) {
    // GetRigidObjectTransform of the Blender animator (start time 0: the
    // reference leaves _timeStart unset for it)
    int i0 = 0;
    const double u = t / step;
    if (u > 0) i0 = u >= (double)n ? n - 1 : (int)u;
    i0 = std::min(std::max(0, i0), n - 1);
    const int i1 = std::min(i0 + 1, n - 1);
    const double t0 = i0 * step, t1 = i1 * step;
    const double alpha = i0 == i1 ? 1.0 : (t - t0) / (t1 - t0);
    const double* f0 = frames + 7 * (size_t)i0;
    const double* f1 = frames + 7 * (size_t)i1;
    for (int d = 0; d < 3; ++d) com[d] = f0[d] * (1.0 - alpha) + f1[d] * alpha;
    Quat q = slerp({f0[3], f0[4], f0[5], f0[6]}, alpha, {f1[3], f1[4], f1[5], f1[6]});
    normalize(q);  // FDTD_Objects::AnimateObjects
    rotation_matrix(q, R);
}

bool read_kinematics(const char* path, std::vector<double>& frames, std::string& err) {
    std::ifstream f(path);
    if (!f) {
        err = std::string("cannot open kinematics file ") + path;
        return false;
    }
    // -90 degrees about x: Quaternion::fromAxisRotD((1, 0, 0), -90)
    const double half = (-90.0 * M_PI / 180.0) / 2;
    const Quat corr{std::cos(half), 1.0 * std::sin(half), 0.0 * std::sin(half), 0.0 * std::sin(half)};
    std::string line;
    frames.clear();
    while (std::getline(f, line)) {
        std::istringstream is(line);
        double fr, v[7];
        if (!(is >> fr)) continue;
        for (int k = 0; k < 7; ++k)
            if (!(is >> v[k])) {
                err = std::string("kinematics file ") + path + ": a line needs 8 numbers";
                return false;
            }
        const double w = std::max(-1.0, std::min(1.0, v[3]));
        const Quat q = mul(Quat{w, v[4], v[5], v[6]}, corr);
        frames.insert(frames.end(), {v[0], v[1], v[2], q.w, q.x, q.y, q.z});
    }
    if (frames.empty()) {
        err = std::string("kinematics file ") + path + " has no frame";
        return false;
    }
    return true;
}

}  // namespace fdtd

extern "C" {

fdtd_status fdtd_read_kinematics(const char* path, int32_t* n_frames, double* frames, int64_t capacity) {
    if (!path || !n_frames) return (fdtd::set_error(nullptr, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    std::vector<double> fr;
    std::string err;
    if (!fdtd::read_kinematics(path, fr, err)) return (fdtd::set_error(nullptr, err), FDTD_ERR_IO);
    *n_frames = (int32_t)(fr.size() / 7);
    if (!frames) return FDTD_OK;
    if (capacity < (int64_t)fr.size()) return (fdtd::set_error(nullptr, "frames buffer too small"), FDTD_ERR_INVALID_ARG);
    std::copy(fr.begin(), fr.end(), frames);
    return FDTD_OK;
}

fdtd_status fdtd_keyframe_pose(const fdtd_keyframe_track* track, double t, double* com, double* rotation) {
    if (!track || !track->frames || track->n_frames < 1 || !(track->step > 0) || !com || !rotation)
        return (fdtd::set_error(nullptr, "invalid keyframe track"), FDTD_ERR_INVALID_ARG);
    fdtd::keyframe_pose(track->frames, track->n_frames, track->step, t, com, rotation);
    return FDTD_OK;
}

}  // extern "C"
