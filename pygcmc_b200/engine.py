"""Device-resident GCMC contexts over the C ABI (gcmc_create ... gcmc_destroy).

An :class:`Engine` holds one or more independent replicas on the GPU and
advances them together; each MC step is one launch of the pose-energy kernel
(all replicas' trial poses) and one of the accept kernel (one CTA per
replica), replayed from a captured CUDA graph.
"""
import ctypes

import numpy as np

from . import values as V
from ._native import Options, ReplicaIn, TuneTrial, check, default_options, lib, ptr


def _replica_array(systems, options=None):
    arr = (ReplicaIn * len(systems))()
    for i, s in enumerate(systems):
        arr[i] = ReplicaIn(*[ptr(x) for x in s.arrays_for(options)])
    return arr


def autotune(systems, options: Options = None, trial_steps: int = 64):
    """Pick the launch shape (cell-grid resolution, pose-energy work split,
    graph branches, pose-energy CTAs per SM) for these replicas by timing
    short runs on temporary contexts (gcmc_autotune).  Returns the options to
    create the :class:`Engine` with and the list of trials
    ``(cells_per_cutoff, split_items, branches, energy_blocks_per_sm, energy_variant, ms_per_step,
    energy_kernel, tile_cells, persistent)``."""
    if not isinstance(systems, (list, tuple)):
        systems = [systems]
    base = options if options is not None else default_options()
    arr = _replica_array(systems, base)
    best = Options()
    trials = (TuneTrial * 32)()
    n = ctypes.c_int32(0)
    check(lib().gcmc_autotune(len(systems), arr, ctypes.byref(base), int(trial_steps), ctypes.byref(best), trials,
                              32, ctypes.byref(n)), "gcmc_autotune")
    out = [(t.cells_per_cutoff, t.split_items, t.branches, t.energy_blocks_per_sm, t.energy_variant,
            float(t.ms_per_step), t.energy_kernel, t.tile_cells, t.persistent) for t in trials[: min(n.value, 32)]]
    return best, out


class Engine:
    def __init__(self, systems, options: Options = None, stream=None):
        """``systems``: a :class:`pygcmc_b200.system.System` or a list of them.
        ``stream``: an integer cudaStream_t (e.g. ``torch.cuda.Stream().cuda_stream``)
        or None for a library-owned stream."""
        if not isinstance(systems, (list, tuple)):
            systems = [systems]
        self.systems = list(systems)
        self.options = options if options is not None else default_options()
        arr = _replica_array(self.systems, self.options)
        self._in = arr
        h = ctypes.c_void_p()
        check(lib().gcmc_create(len(self.systems), arr, ctypes.byref(self.options),
                                ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)), "gcmc_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return lib().gcmc_stream(self._h) or 0

    def run(self, nsteps: int):
        check(lib().gcmc_run(self._h, int(nsteps)), "gcmc_run")

    def run_profiled(self, nsteps: int):
        """Run nsteps with per-step kernel timing; returns (ms_energy, ms_accept, move)."""
        n = int(nsteps)
        te = np.zeros(n, np.float32)
        ta = np.zeros(n, np.float32)
        mv = np.zeros(n, np.int32)
        check(lib().gcmc_run_profiled(self._h, n, ptr(te), ptr(ta), ptr(mv)), "gcmc_run_profiled")
        return te, ta, mv

    def sync(self):
        check(lib().gcmc_sync(self._h), "gcmc_sync")

    def download(self, rep: int = 0, into=None):
        """Replica state as (fragmentInfo, residueInfo, atomInfo); copies of the
        inputs updated in place unless ``into`` (a System) is given."""
        s = into if into is not None else self.systems[rep].copy()
        check(lib().gcmc_download(self._h, rep, ptr(s.fragmentInfo), ptr(s.residueInfo), ptr(s.atomInfo)),
              "gcmc_download")
        return s

    def checkpoint(self, rep: int = 0):
        """The replica's state after the steps run so far, as a System whose
        move schedule is the remaining steps; ``meta["step_offset"]`` is the
        absolute step to resume at (pass it as ``options.step_offset`` when
        creating the Engine that continues the chain)."""
        c = self.counters(rep)
        done = int(c["steps"]) if c["steps"] >= 0 else 0
        base = int(self.systems[rep].meta.get("step_offset", 0))
        s = self.download(rep)
        s.moveArray = np.ascontiguousarray(self.systems[rep].moveArray[done:])
        s.SimInfo = s.SimInfo.copy()
        s.SimInfo[0]["mcsteps"] = len(s.moveArray)
        s.meta = dict(s.meta)
        s.meta["step_offset"] = base + done
        return s

    def logs(self, rep: int = 0):
        n = int(self.options.log_steps)
        logs = np.zeros(n, dtype=V.StepLog_dtype)
        E = np.zeros((n, max(1, int(self.options.log_kmax))), dtype=np.float64)
        got = ctypes.c_int32(0)
        check(lib().gcmc_get_logs(self._h, rep, ptr(logs), ptr(E), n, ctypes.byref(got)), "gcmc_get_logs")
        return logs[: got.value], E[: got.value]

    def forces(self, rep: int = 0):
        """Force-biased runs with logs: [steps, log_kmax, 12] float32 -- old-pose
        force and torque, then new-pose force and torque, of each pose."""
        n = int(self.options.log_steps)
        km = max(1, int(self.options.log_kmax))
        out = np.zeros((n, km, 12), dtype=np.float32)
        got = ctypes.c_int32(0)
        check(lib().gcmc_get_forces(self._h, rep, ptr(out), n, ctypes.byref(got)), "gcmc_get_forces")
        return out[: got.value]

    def pme_potential(self, pts, rep: int = 0):
        """Ewald runs: reciprocal-space potential (kJ/mol/e) of the current state at points [n, 3]."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(len(pts))
        check(lib().gcmc_pme_potential(self._h, rep, ptr(pts), len(pts), ptr(out)), "gcmc_pme_potential")
        return out

    def energy_total(self, rep: int = 0) -> float:
        """Running sum of the accepted energy changes since creation (kJ/mol)."""
        e = ctypes.c_double(0.0)
        check(lib().gcmc_energy_total(self._h, rep, ctypes.byref(e)), "gcmc_energy_total")
        return e.value

    def counters(self, rep: int = 0):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().gcmc_counters(self._h, rep, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "gcmc_counters")
        return {"steps": a.value, "poses": b.value, "pairs": c.value}

    def phase_cycles(self, rep: int = 0):
        """Accept-kernel SM cycles per phase (energies, precompute, cluster walk,
        update, prepare), the number of speculative cluster rounds and the
        number of steps whose pose energies were evaluated beside the previous
        step's accept kernel and kept."""
        out = np.zeros(8, np.int64)
        check(lib().gcmc_phase_cycles(self._h, rep, ptr(out)), "gcmc_phase_cycles")
        return out[:7]

    def device_error(self) -> int:
        e = ctypes.c_int32(0)
        check(lib().gcmc_device_error(self._h, ctypes.byref(e)), "gcmc_device_error")
        return e.value

    def energy_poses(self, xyz, q, types, centres, self_res=None, rep: int = 0):
        """Energies (kJ/mol, FP64 sums of FP32 pair terms) of explicit poses and
        the number of groups inside the cutoff of each."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        n, ns = xyz.shape[0], xyz.shape[1]
        q = np.ascontiguousarray(q, dtype=np.float32)
        t = np.ascontiguousarray(types, dtype=np.int32)
        c = np.ascontiguousarray(centres, dtype=np.float32)
        sr = None if self_res is None else np.ascontiguousarray(self_res, dtype=np.int32)
        out = np.zeros(n, dtype=np.float64)
        ng = np.zeros(n, dtype=np.int32)
        check(lib().gcmc_energy_poses(self._h, rep, ptr(xyz), ptr(q), ptr(t), ns, ptr(c), ptr(sr), n, ptr(out),
                                      ptr(ng)), "gcmc_energy_poses")
        return out, ng

    def close(self):
        if getattr(self, "_h", None):
            lib().gcmc_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
