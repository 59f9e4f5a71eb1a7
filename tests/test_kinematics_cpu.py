"""Keyframed rigid-body poses (host side): the library's pose query against an
independent numpy restatement of the reference's animator
(FDTD_RigidObject_Animator.cpp:79-155, Quaternion.hpp:186-208, :298-313,
:392-420, FDTD_RigidObject.cpp:549-566); the kinematics-file reader with its
y-up correction; the XML attribute that loads it; the oracle stepping a
keyframed scene."""
import ctypes as C
import math

import numpy as np
import pytest

from acoustics_b200 import scene as S


# ---- numpy restatement ------------------------------------------------------
def q_norm(q):
    q = np.asarray(q, dtype=np.float64).copy()
    n2 = q[0] * q[0] + (q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    if abs(n2 - 1.0) > 1e-12:
        q = q * (1.0 / math.sqrt(n2))
    return q


def q_mul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 + y1 * w2 + z1 * x2 - x1 * z2, w1 * z2 + z1 * w2 + x1 * y2 - y1 * x2])


def q_slerp(q0, r, q1):
    v0, v1 = q_norm(q0), q_norm(q1)
    d = float(np.dot(v0, v1))
    if abs(d) > 0.9995:
        return q_norm(v0 + (v1 - v0) * r)
    if d < 0:
        v1, d = -v1, -d
    d = min(max(d, -1.0), 1.0)
    th = math.acos(d) * r
    v2 = q_norm(v1 - v0 * d)
    return v0 * math.cos(th) + v2 * math.sin(th)


def rot_from_quat(q):
    ang = 2.0 * math.acos(q[0])
    a = np.array([0.0, 1.0, 0.0]) if ang < 1e-12 else np.asarray(q[1:]) / np.linalg.norm(q[1:])
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return math.cos(ang) * np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * np.outer(a, a)


def pose(frames, step, t):
    n = len(frames)
    u = t / step
    i0 = 0 if u <= 0 else min(int(u), n - 1)
    i1 = min(i0 + 1, n - 1)
    al = 1.0 if i0 == i1 else (t - i0 * step) / (i1 * step - i0 * step)
    com = frames[i0][:3] * (1 - al) + frames[i1][:3] * al
    q = q_norm(q_slerp(frames[i0][3:], al, frames[i1][3:]))
    return com, rot_from_quat(q)


def random_track(rng, n, close=False):
    fr = np.zeros((n, 7))
    q = q_norm(rng.normal(size=4))
    for i in range(n):
        fr[i, :3] = rng.uniform(-0.05, 0.05, 3)
        if i > 0:
            dq = q_norm(np.r_[1.0, rng.normal(scale=0.001 if close else 0.6, size=3)])
            q = q_norm(q_mul(q, dq))
            if rng.uniform() < 0.3:
                q = -q  # the same rotation from the other hemisphere: the slerp flips it
        fr[i, 3:] = q
    return fr


def lib_pose(lib, frames, step, t):
    fr = np.ascontiguousarray(frames, dtype=np.float64)
    tr = S.KeyframeTrackDesc(0, fr.shape[0], step, fr.ctypes.data_as(C.POINTER(C.c_double)))
    com, R = np.zeros(3), np.zeros(9)
    assert lib.fdtd_keyframe_pose(C.byref(tr), float(t), com.ctypes.data, R.ctypes.data) == 0
    return com, R.reshape(3, 3)


@pytest.mark.parametrize("close", [False, True])
def test_pose_matches_restatement(fdtd_lib, close):
    rng = np.random.default_rng(3 if close else 4)
    fr = random_track(rng, 9, close)
    step = 1.0 / 30.0
    for t in np.concatenate([[-0.1, 0.0], rng.uniform(0, 9 * step, 200), [8 * step, 8.5 * step, 1.0]]):
        c1, R1 = lib_pose(fdtd_lib, fr, step, t)
        c2, R2 = pose(fr, step, t)
        assert np.allclose(c1, c2, rtol=0, atol=1e-15), t
        assert np.allclose(R1, R2, rtol=0, atol=1e-13), t
        assert np.allclose(R1 @ R1.T, np.eye(3), atol=1e-13)


def test_read_kinematics_applies_the_y_up_turn(fdtd_lib, tmp_path):
    rng = np.random.default_rng(7)
    rows = []
    for f in range(5):
        q = q_norm(rng.normal(size=4))
        rows.append([f, *rng.uniform(-1, 1, 3), *q])
    rows[2][4] = 1.5  # w is clamped to 1
    p = tmp_path / "obj.kin"
    p.write_text("\n".join(" ".join(repr(float(v)) for v in r) for r in rows) + "\n")
    n = C.c_int32(0)
    assert fdtd_lib.fdtd_read_kinematics(str(p).encode(), C.byref(n), None, 0) == 0 and n.value == 5
    out = np.zeros((5, 7))
    assert fdtd_lib.fdtd_read_kinematics(str(p).encode(), C.byref(n), out.ctypes.data, out.size) == 0
    half = math.radians(-90.0) / 2
    corr = np.array([math.cos(half), math.sin(half), 0.0, 0.0])
    for r, o in zip(rows, out):
        q = np.array([min(1.0, max(-1.0, r[4])), r[5], r[6], r[7]])
        assert np.allclose(o[:3], r[1:4], rtol=0, atol=0)
        assert np.allclose(o[3:], q_mul(q, corr), rtol=0, atol=1e-16)


def keyframed_scene(n=40, steps=60):
    """A box turning a quarter turn about z and a sphere moving on keyframes (30 Hz
    frames stretched so the motion spans the run), a source and listeners."""
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=(n, n, n), time_step=S.reference_time_step(h), pml_width=6, steps=steps,
                 name="keyframed")
    step = steps * sc.time_step / 4  # four frame intervals over the run
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.0, 0.0, 0.0), (0.03, 0.012, 0.01), motion=S.MOTION_KEYFRAMED))
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.0, 0.0, 0.0), (0.012, 0, 0), motion=S.MOTION_KEYFRAMED))
    box = np.zeros((5, 7))
    sph = np.zeros((5, 7))
    for i in range(5):
        a = math.radians(22.5 * i)
        box[i] = [0.002 * i, -0.01, 0.0, math.cos(a / 2), 0.0, 0.0, math.sin(a / 2)]
        sph[i] = [0.0, 0.04 - 0.004 * i, 0.01 * math.sin(i), 1.0, 0.0, 0.0, 0.0]
    sc.tracks = [S.KeyframeTrack(0, step, box), S.KeyframeTrack(1, step, sph)]
    sc.sources.append(S.GaussianSource((-0.04, 0.0, 0.03), 5e-5))
    sc.listeners = np.array([[0.045, 0.0, 0.0], [0.0, -0.045, 0.01], [-0.03, 0.03, -0.03]])
    return sc


def test_xml_file_kinematics(fdtd_lib, tmp_path):
    from acoustics_b200.solver import scene_from_xml
    (tmp_path / "box.kin").write_text("0 0 0 0 1 0 0 0\n1 0.01 0 0 0.7071067811865476 0.7071067811865476 0 0\n")
    (tmp_path / "scene.xml").write_text("""<?xml version="1.0" ?>
<impulse_response>
  <solver cellsize="0.005" timestepfrequency="118800" PML_width="6" PML_strength="1e6" number_of_timesteps="10"/>
  <solver_control_policy type="static" gridresolution="40"/>
  <scene>
    <analytic_box center_x="0" center_y="0" center_z="0" half_x="0.02" half_y="0.01" half_z="0.01"
                  file_kinematics="box.kin" kinematics_frame_rate="30"/>
  </scene>
  <listening_point_list><listening_point x="0.05" y="0" z="0"/></listening_point_list>
</impulse_response>
""")
    sc = scene_from_xml(str(tmp_path / "scene.xml"))
    assert sc.objects[0].motion == S.MOTION_KEYFRAMED
    assert len(sc.tracks) == 1 and sc.tracks[0].object == 0 and abs(sc.tracks[0].step - 1 / 30) < 1e-15
    assert sc.tracks[0].frames.shape == (2, 7)


def test_oracle_steps_a_keyframed_scene(oracle_lib):
    sc = keyframed_scene()
    o = oracle_lib.OracleSolver(sc)
    y = o.step(sc.steps)
    assert np.isfinite(y).all() and np.abs(y).max() > 0
    flags, faces = o.classification()
    assert len(faces) > 0
