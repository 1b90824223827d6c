"""Rigid fragment poses: centre of mass + unit quaternion -> site coordinates.

A pose of fragment type f places the type's template (its AtomArray sites,
centred on their centroid) rotated by the quaternion q = (w, x, y, z) and
translated to the centre of mass c:  x_s = c + R(q) (t_s - t_mean).  The
group-inclusion centre of the pose is c (the unweighted site centroid, as the
reference uses for fragment residues, dataset.py:248-275).
"""
import numpy as np


def template(system, ftype: int):
    """(centred template sites [ns, 3] float64, charges [ns] float32, types [ns] int32)."""
    f = system.fragmentInfo[ftype]
    ns = int(f["num_atoms"])
    t = f["atoms"]["position"][:ns].astype(np.float64)
    return (t - t.mean(axis=0), f["atoms"]["charge"][:ns].astype(np.float32).copy(),
            f["atoms"]["type"][:ns].astype(np.int32).copy())


def quat_to_matrix(q):
    """Rotation matrices [n, 3, 3] of unit quaternions q [n, 4] = (w, x, y, z)."""
    q = np.asarray(q, dtype=np.float64)
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    w, x, y, z = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def rigid_sites(tpl, com, quat):
    """Site coordinates [n, ns, 3] (float64) of poses (com [n, 3], quat [n, 4])."""
    R = quat_to_matrix(quat)
    return np.asarray(com, dtype=np.float64)[:, None, :] + np.einsum("nij,sj->nsi", R, tpl)


def random_poses(system, n: int, seed: int = 0):
    """n poses with the centre of mass uniform in the box and a uniform random
    quaternion (Shoemake); returns (com [n, 3], quat [n, 4]) float64."""
    g = np.random.default_rng(seed)
    info = system.SimInfo[0]
    lo = np.asarray(info["startxyz"], dtype=np.float64)
    L = np.asarray(info["cryst"], dtype=np.float64)
    com = lo + g.random((n, 3)) * L
    u1, u2, u3 = g.random(n), 2 * np.pi * g.random(n), 2 * np.pi * g.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    quat = np.stack([b * np.cos(u3), a * np.sin(u2), a * np.cos(u2), b * np.sin(u3)], -1)
    return com, quat
