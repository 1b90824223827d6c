"""ctypes binding of the native library's C ABI (include/gcmc_b200.h).

The library is built in-tree by :mod:`pygcmc_b200.build`; importing this
module never falls back to anything else -- a missing library raises.
"""
import ctypes
import os

import numpy as np

from .build import LIB_PATH

c_int = ctypes.c_int32
c_void = ctypes.c_void_p


class Options(ctypes.Structure):
    """gcmc_options (include/gcmc_b200.h)."""
    _fields_ = [("proposal", c_int), ("muex_kcal", c_int), ("trn_step", ctypes.c_float),
                ("rot_max", ctypes.c_float), ("replica", ctypes.c_uint32), ("cells_per_cutoff", c_int),
                ("log_steps", c_int), ("log_kmax", c_int), ("split_items", c_int), ("branches", c_int),
                ("energy_blocks_per_sm", c_int), ("fb_trn", ctypes.c_float), ("fb_rot", ctypes.c_float),
                ("step_offset", ctypes.c_uint32), ("pme", c_int), ("pme_alpha", ctypes.c_float),
                ("pme_grid", c_int * 3), ("energy_variant", c_int), ("speculate", c_int),
                ("energy_kernel", c_int), ("tile_cells", c_int), ("pair_delta", c_int),
                ("persistent", c_int), ("persist_spin_cap", c_int), ("pose_split", c_int),
                ("grid_bits", c_int)]


class TuneTrial(ctypes.Structure):
    """gcmc_tune_trial: one autotuner trial."""
    _fields_ = [("cells_per_cutoff", c_int), ("split_items", c_int), ("branches", c_int),
                ("energy_blocks_per_sm", c_int), ("energy_variant", c_int), ("ms_per_step", ctypes.c_float),
                ("energy_kernel", c_int), ("tile_cells", c_int), ("persistent", c_int)]


class ReplicaIn(ctypes.Structure):
    """gcmc_replica_in: the seven state arrays of one replica."""
    _fields_ = [("info", c_void), ("fragmentInfo", c_void), ("residueInfo", c_void), ("atomInfo", c_void),
                ("grid", c_void), ("ff", c_void), ("moveArray", c_void)]


STATUS = {0: "ok", 1: "CUDA runtime error", 2: "invalid or inconsistent input",
          3: "a size limit of the engine is exceeded", 4: "the device raised an error flag",
          5: "no CUDA device"}


class GcmcError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'unknown status')} (status {status})")


_lib = None


def lib():
    """The loaded library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"native library missing: {LIB_PATH} (build it with python -m pygcmc_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    sig = {
        "runGCMC_cuda": (None, [c_void] * 7),
        "gcmc_run_gcmc": (c_int, [c_void] * 7 + [P(Options)]),
        "gcmc_last_status": (c_int, []),
        "gcmc_release_cache": (c_int, []),
        "gcmc_pme_potential": (c_int, [c_void, c_int, c_void, c_int, c_void]),
        "gcmc_pdb_fragment_lines": (ctypes.c_int64, [c_int, c_void, c_void, c_void, c_void, ctypes.c_int64,
                                                     ctypes.c_int64, c_void, ctypes.c_int64]),
        "gcmc_cavity_grid": (c_int, [c_int, c_void, c_void, ctypes.c_double, c_int, c_void, c_void, ctypes.c_int64,
                                     P(ctypes.c_int64), P(ctypes.c_double)]),
        "gcmc_cavity_bits": (c_int, [c_int, c_void, c_void, ctypes.c_double, c_int, c_void, c_void, ctypes.c_int64,
                                     P(ctypes.c_int64), P(ctypes.c_int64)]),
        "gcmc_fix_groups": (ctypes.c_int32, [c_int, c_void, ctypes.c_double, c_void]),
        "gcmc_group_centres": (c_int, [c_int, c_void, c_void, c_void, c_void]),
        "gcmc_fill_layout": (c_int, [c_int, c_void, c_void, c_void, c_void, c_int, c_void, c_void, c_void, c_void,
                                     c_void, c_void, c_int, ctypes.c_int64, c_void, c_void, c_void]),
        "gcmc_get_forces": (c_int, [c_void, c_int, c_void, c_int, P(c_int)]),
        "gcmc_energy_total": (c_int, [c_void, c_int, P(ctypes.c_double)]),
        "gcmc_energy_grad": (c_int, [c_void, c_int] + [c_void] * 4 + [c_int, c_void, c_void, c_int] + [c_void] * 7),
        "gcmc_run_batch": (c_int, [c_int, c_void, P(Options)]),
        "gcmc_autotune": (c_int, [c_int, c_void, P(Options), c_int, P(Options), c_void, c_int, P(c_int)]),
        "gcmc_status_string": (ctypes.c_char_p, [c_int]),
        "gcmc_default_options": (None, [P(Options)]),
        "gcmc_create": (c_int, [c_int, P(ReplicaIn), P(Options), c_void, P(c_void)]),
        "gcmc_run": (c_int, [c_void, c_int]),
        "gcmc_sync": (c_int, [c_void]),
        "gcmc_run_profiled": (c_int, [c_void, c_int, c_void, c_void, c_void]),
        "gcmc_download": (c_int, [c_void, c_int, c_void, c_void, c_void]),
        "gcmc_get_logs": (c_int, [c_void, c_int, c_void, c_void, c_int, P(c_int)]),
        "gcmc_counters": (c_int, [c_void, c_int, P(ctypes.c_int64), P(ctypes.c_int64), P(ctypes.c_int64)]),
        "gcmc_device_error": (c_int, [c_void, P(c_int)]),
        "gcmc_phase_cycles": (c_int, [c_void, c_int, c_void]),
        "gcmc_stream": (c_void, [c_void]),
        "gcmc_destroy": (c_int, [c_void]),
        "gcmc_energy_poses": (c_int, [c_void, c_int, c_void, c_void, c_void, c_int, c_void, c_void, c_int,
                                      c_void, c_void]),
        "gcmc_energy_poses_noalloc": (c_int, [c_void, c_int, c_void, c_void, c_void, c_int, c_void, c_void,
                                              c_int, c_void, c_void, c_void]),
        "gcmc_synth_chain_sphere": (c_int, [c_int, c_void, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_uint64, c_void, P(ctypes.c_int)]),
        "gcmc_synth_chain_slab": (c_int, [c_int] + [ctypes.c_float] * 11 + [ctypes.c_uint64, c_void,
                                                                           P(ctypes.c_int)]),
        "gcmc_synth_place": (c_int, [c_int, c_void, c_void, c_void, c_void, c_int, c_int, ctypes.c_float,
                                     ctypes.c_uint64, c_void]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a):
    """Data pointer of a C-contiguous numpy array (None for None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(c_void)


def check(status, what):
    if status != 0:
        raise GcmcError(status, what)


def default_options(**kw):
    o = Options()
    lib().gcmc_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


EXPORTS = ["runGCMC_cuda", "gcmc_run_gcmc", "gcmc_run_batch", "gcmc_energy_grad", "gcmc_get_forces", "gcmc_pme_potential",
           "gcmc_cavity_grid", "gcmc_cavity_bits", "gcmc_fix_groups", "gcmc_group_centres", "gcmc_fill_layout", "gcmc_pdb_fragment_lines",
           "gcmc_energy_total", "gcmc_autotune", "gcmc_release_cache", "gcmc_last_status", "gcmc_status_string", "gcmc_default_options",
           "gcmc_create", "gcmc_run", "gcmc_run_profiled", "gcmc_sync", "gcmc_download", "gcmc_get_logs", "gcmc_counters",
           "gcmc_device_error", "gcmc_phase_cycles", "gcmc_stream", "gcmc_destroy", "gcmc_energy_poses",
           "gcmc_energy_poses_noalloc", "gcmc_synth_place", "gcmc_synth_chain_sphere",
           "gcmc_synth_chain_slab"]
