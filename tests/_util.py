import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def small_config2(n=80, steps=150):
    """Configuration 2 geometry (sphere, box, ellipsoid with Gaussian translational
    boundary acceleration) on a reduced grid with a coarser cell so the bodies fit."""
    from acoustics_b200 import scene as S
    sc = S.config2()
    sc.divisions = (n, n, n)
    sc.cell_size = 0.0025 * 256 / n * 0.5
    sc.time_step = S.reference_time_step(sc.cell_size)
    sc.pml_width = 8
    for o in sc.objects:
        o.center = tuple(np.asarray(o.center) * 0.5)
        o.size = tuple(np.asarray(o.size) * 0.5)
        o.accel_tau = 40 * sc.time_step
        o.accel_t0 = 4 * o.accel_tau
    sc.listeners = np.asarray(sc.listeners) * 0.5
    sc.steps = steps
    return sc


def small_scene_with(*objects, meshes=(), n=40, steps=20):
    """A small static scene (n^3, h = 5 mm, PML 6) with the given objects and
    meshes, one source and two listeners away from the domain centre."""
    from acoustics_b200 import scene as S
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=(n, n, n), time_step=S.reference_time_step(h), pml_width=6, steps=steps,
                 name="small_with_objects")
    sc.objects.extend(objects)
    sc.meshes.extend(meshes)
    sc.sources.append(S.GaussianSource((0.0, 0.06, 0.0), 1e-4))
    sc.listeners = np.array([[0.0, -0.06, 0.01], [0.05, 0.0, -0.02]])
    return sc
