"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this module; it checks the engine and is never part of it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
c_void = ctypes.c_void_p


class OrOptions(ctypes.Structure):
    _fields_ = [("proposal", ctypes.c_int32), ("muex_kcal", ctypes.c_int32), ("trn_step", ctypes.c_float),
                ("rot_max", ctypes.c_float), ("replica", ctypes.c_uint32), ("fb_trn", ctypes.c_float),
                ("fb_rot", ctypes.c_float), ("pme", ctypes.c_int32), ("pme_alpha", ctypes.c_float)]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.or_run_ext.restype = ctypes.c_int32
        L.or_run_ext.argtypes = [c_void] * 8 + [ctypes.c_int32, ctypes.c_int32, c_void, c_void, c_void, c_void,
                                                ctypes.c_int32, ctypes.c_int32, c_void, c_void, c_void, c_void]
        L.or_decision_stats.restype = None
        L.or_decision_stats.argtypes = [ctypes.c_int32, c_void, c_void, c_void]
        L.or_det_log.restype = ctypes.c_float
        L.or_det_log.argtypes = [ctypes.c_float]
        L.or_ewald_potential.argtypes = [c_void] * 4 + [ctypes.c_double, c_void, ctypes.c_int32, c_void,
                                                        ctypes.c_int32]
        L.or_det_exp_neg.restype = ctypes.c_float
        L.or_det_exp_neg.argtypes = [ctypes.c_float]
        L.or_run.restype = ctypes.c_int32
        L.or_run.argtypes = [c_void] * 8 + [ctypes.c_int32, ctypes.c_int32, c_void, c_void, c_void, c_void,
                                            ctypes.c_int32, ctypes.c_int32]
        L.or_energy_batch.restype = ctypes.c_int64
        L.or_energy_batch.argtypes = [c_void] * 8 + [ctypes.c_int32, c_void, c_void, ctypes.c_int32, ctypes.c_int32,
                                                     c_void, c_void, c_void, ctypes.c_int32]
        L.or_energy_batch64.restype = ctypes.c_int64
        L.or_energy_batch64.argtypes = [c_void] * 7 + [c_void, ctypes.c_int32, c_void, c_void, ctypes.c_int32,
                                                       c_void, c_void, ctypes.c_int32]
        L.or_grad_batch.restype = ctypes.c_int64
        L.or_grad_batch.argtypes = [c_void] * 7 + [c_void, ctypes.c_int32, c_void, c_void, ctypes.c_int32] + \
            [c_void] * 7 + [ctypes.c_int32]
        L.or_philox.argtypes = [c_void, c_void, c_void]
        L.or_det_sincos.argtypes = [ctypes.c_float, c_void, c_void]
        L.or_dist_group.restype = ctypes.c_float
        L.or_dist_group.argtypes = [c_void, c_void, c_void]
        L.or_dist_host.restype = ctypes.c_float
        L.or_dist_host.argtypes = [c_void, c_void, c_void]
        L.or_insert_pose.argtypes = [c_void, c_void, c_void, c_void, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                     c_void, c_void]
        L.or_move_pose.argtypes = [c_void] * 5 + [ctypes.c_int32] * 5 + [c_void, c_void]
        L.or_rotate_point.argtypes = [c_void, ctypes.c_float, c_void, c_void, c_void]
        L.or_perm_slot.restype = ctypes.c_int32
        L.or_perm_slot.argtypes = [c_void, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void)


def options(proposal=0, muex_kcal=0, trn_step=1.0, rot_max=np.radians(15.0), replica=0, fb_trn=0.5,
            fb_rot=np.radians(10.0), pme=0, pme_alpha=0.32):
    return OrOptions(proposal, muex_kcal, trn_step, rot_max, replica, fb_trn, fb_rot, pme, pme_alpha)


def ewald_potential(system, alpha, pts, threads=None):
    """Exact Ewald reciprocal-space potential (kJ/mol/e) of the state at points [n, 3]."""
    threads = threads or os.cpu_count() or 1
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(pts))
    s = system
    lib().or_ewald_potential(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), float(alpha),
                             _p(pts), len(pts), _p(out), threads)
    return out


def decision_stats(reset=True):
    """(decisions, decisions within the per-trial tolerance band of their
    threshold, smallest margin / tolerance) since the last reset."""
    t, b, m = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
    lib().or_decision_stats(1 if reset else 0, ctypes.byref(t), ctypes.byref(b), ctypes.byref(m))
    return t.value, b.value, m.value


def run_ext(system, nsteps, step0=0, opts=None, kmax=1024, threads=None, replay=None, replay_forces=None,
            e_total=0.0):
    """:func:`run` with the running energy and the force-biased extensions.
    Returns a dict: logs, energies, scale, forces [n, kmax, 12] (the oracle's
    FP64 old/new force and torque of force-biased poses), fscale [n, kmax, 4]
    and e_total (the running energy after the last step)."""
    from pygcmc_b200.values import StepLog_dtype
    opts = opts or options()
    threads = threads or os.cpu_count() or 1
    out = {"logs": np.zeros(nsteps, dtype=StepLog_dtype), "energies": np.zeros((nsteps, kmax)),
           "scale": np.zeros((nsteps, kmax)), "forces": np.zeros((nsteps, kmax, 12)),
           "fscale": np.zeros((nsteps, kmax, 4))}
    rp = None if replay is None else np.ascontiguousarray(replay, dtype=np.float64)
    rf = None if replay_forces is None else np.ascontiguousarray(replay_forces, dtype=np.float32)
    et = ctypes.c_double(e_total)
    s = system
    rc = lib().or_run_ext(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), _p(s.grid),
                          _p(s.ff), _p(s.moveArray), ctypes.byref(opts), step0, nsteps, _p(out["logs"]),
                          _p(out["energies"]), _p(out["scale"]), _p(rp), kmax, threads, ctypes.byref(et),
                          _p(out["forces"]), _p(out["fscale"]), _p(rf))
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
    out["e_total"] = et.value
    return out



def run(system, nsteps, step0=0, opts=None, kmax=1024, threads=None, replay=None, want_energies=True,
        want_scale=False):
    """Advance a System in place; returns (logs, energies) or, with want_scale,
    (logs, energies, scale) where scale is the magnitude the relative tolerance
    of each energy refers to (|E|, or |E_new| + |E_old| for translate/rotate)."""
    from pygcmc_b200.values import StepLog_dtype
    opts = opts or options()
    threads = threads or os.cpu_count() or 1
    logs = np.zeros(nsteps, dtype=StepLog_dtype)
    E = np.zeros((nsteps, kmax), dtype=np.float64) if want_energies else None
    SC = np.zeros((nsteps, kmax), dtype=np.float64) if want_scale else None
    rp = None if replay is None else np.ascontiguousarray(replay, dtype=np.float64)
    s = system
    rc = lib().or_run(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), _p(s.grid), _p(s.ff),
                      _p(s.moveArray), ctypes.byref(opts), step0, nsteps, _p(logs), _p(E), _p(SC), _p(rp), kmax,
                      threads)
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
    return (logs, E, SC) if want_scale else (logs, E)


def energy_batch(system, xyz, q, types, centres, self_res=None, mode=0, threads=None, want_l1=False):
    """FP64 (mode 0) or FP32-mirror (mode 1) energies of explicit poses:
    (energies, groups included, pairs) and, with want_l1, the per-pose sum of
    |pair terms| (FP64 mode)."""
    threads = threads or os.cpu_count() or 1
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    n, ns = xyz.shape[0], xyz.shape[1]
    q = np.ascontiguousarray(q, dtype=np.float32)
    t = np.ascontiguousarray(types, dtype=np.int32)
    c = np.ascontiguousarray(centres, dtype=np.float32)
    sr = None if self_res is None else np.ascontiguousarray(self_res, dtype=np.int32)
    out = np.zeros(n, dtype=np.float64)
    ng = np.zeros(n, dtype=np.int32)
    l1 = np.zeros(n, dtype=np.float64)
    s = system
    pairs = lib().or_energy_batch(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), _p(s.ff),
                                  _p(xyz), _p(q), _p(t), ns, _p(c), _p(sr), n, mode, _p(out), _p(ng), _p(l1),
                                  threads)
    return (out, ng, int(pairs), l1) if want_l1 else (out, ng, int(pairs))


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().or_philox(_p(c), _p(k), _p(o))
    return o


def det_sincos(x):
    s, c = np.zeros(1, np.float32), np.zeros(1, np.float32)
    lib().or_det_sincos(ctypes.c_float(x), _p(s), _p(c))
    return float(s[0]), float(c[0])


def insert_pose(system, ftype, step, i, opts=None):
    opts = opts or options()
    ns = int(system.fragmentInfo[ftype]["num_atoms"])
    xyz = np.zeros((20, 3), np.float32)
    c = np.zeros(3, np.float32)
    lib().or_insert_pose(_p(system.SimInfo), _p(system.fragmentInfo), _p(system.grid), ctypes.byref(opts), ftype,
                         step, i, _p(xyz), _p(c))
    return xyz[:ns], c


def rotate_point(axis, angle, p):
    a = np.asarray(axis, np.float32)
    x = np.asarray(p, np.float32)
    out = np.zeros(3, np.float32)
    R = np.zeros(9, np.float32)
    lib().or_rotate_point(_p(a), ctypes.c_float(angle), _p(x), _p(out), _p(R))
    return out, R.reshape(3, 3)


def energy_batch64(system, xyz, q, types, centres, ff=None, self_res=None, threads=None):
    """FP64 energies of poses given by FP64 sites ``xyz[P, ns, 3]``, FP64 site
    charges ``q[ns]`` and an FP64 pair table ``ff`` (default: the system's)."""
    threads = threads or os.cpu_count() or 1
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n, ns = xyz.shape[0], xyz.shape[1]
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(types, dtype=np.int32)
    c = np.ascontiguousarray(centres, dtype=np.float32)
    f = np.ascontiguousarray(system.ff if ff is None else ff, dtype=np.float64)
    sr = None if self_res is None else np.ascontiguousarray(self_res, dtype=np.int32)
    out = np.zeros(n, dtype=np.float64)
    ng = np.zeros(n, dtype=np.int32)
    s = system
    lib().or_energy_batch64(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), _p(f), _p(xyz),
                            _p(q), _p(t), ns, _p(c), _p(sr), n, _p(out), _p(ng), threads)
    return out, ng


def grad_batch(system, xyz, q, types, centres, ff=None, self_res=None, gout=None, threads=None):
    """FP64 analytic gradients of :func:`energy_batch64`: returns a dict with
    gxyz [P, ns, 3], gq [P, ns], gff [ffX*ffY*2] (weighted by gout) and their
    l1 scales gxyz_l1 [P, ns], gq_l1 [P, ns], gff_l1."""
    threads = threads or os.cpu_count() or 1
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n, ns = xyz.shape[0], xyz.shape[1]
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(types, dtype=np.int32)
    c = np.ascontiguousarray(centres, dtype=np.float32)
    f = np.ascontiguousarray(system.ff if ff is None else ff, dtype=np.float64)
    sr = None if self_res is None else np.ascontiguousarray(self_res, dtype=np.int32)
    go = None if gout is None else np.ascontiguousarray(gout, dtype=np.float64)
    r = {"gxyz": np.zeros((n, ns, 3)), "gq": np.zeros((n, ns)), "gff": np.zeros(len(f)),
         "gxyz_l1": np.zeros((n, ns)), "gq_l1": np.zeros((n, ns)), "gff_l1": np.zeros(len(f))}
    s = system
    rc = lib().or_grad_batch(_p(s.SimInfo), _p(s.fragmentInfo), _p(s.residueInfo), _p(s.atomInfo), _p(f), _p(xyz),
                             _p(q), _p(t), ns, _p(c), _p(sr), n, _p(go), _p(r["gxyz"]), _p(r["gq"]), _p(r["gff"]),
                             _p(r["gxyz_l1"]), _p(r["gq_l1"]), _p(r["gff_l1"]), threads)
    if rc != 0:
        raise MemoryError("or_grad_batch")
    return r
