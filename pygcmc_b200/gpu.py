"""Drop-in replacement of pyGCMC's native module ``gcmc.gpu``.

``runGCMC(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray)``
has the signature, argument meaning and in-place semantics of the reference
binding (gcmc/cpp/gcmc.cpp:162-197, called from gcmc/python/gcmc.py:41-49):
it runs ``SimInfo[0]['mcsteps']`` steps of ``moveArray`` and writes
``fragmentInfo['totalNum']``, ``residueInfo`` and ``atomInfo`` back in place,
returning ``None``.  Unlike the reference it checks the arrays first and raises
(``TypeError``/``ValueError`` for bad arrays, :class:`GcmcError` for engine
failures) instead of running on undefined input.
"""
import numpy as np

from . import values as V
from ._native import GcmcError, check, default_options, lib, ptr

__all__ = ["runGCMC", "GcmcError", "validate_arrays"]


GRID_BITS_HEADER = 48  # sizeof(gcmc_grid_bits)


def grid_bits_size(rec) -> int:
    """Bytes a gcmc_grid_bits record needs: the header plus ceil(voxels / 32) words."""
    if rec.size < GRID_BITS_HEADER:
        raise ValueError(f"grid holds {rec.size} bytes, a gcmc_grid_bits header needs {GRID_BITS_HEADER}")
    n = np.frombuffer(rec[32:44].tobytes(), dtype=np.int32)
    if (n < 1).any():
        raise ValueError("gcmc_grid_bits: voxel counts must be >= 1")
    return GRID_BITS_HEADER + 4 * ((int(n[0]) * int(n[1]) * int(n[2]) + 31) // 32)


def validate_arrays(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray, grid_bits=False):
    """Dtype, contiguity and size checks against the sizes recorded in SimInfo
    (``grid_bits``: ``grid`` is a uint8 gcmc_grid_bits record instead of the
    float list)."""
    spec = [("SimInfo", SimInfo, V.Info_dtype), ("fragmentInfo", fragmentInfo, V.AtomArray_dtype),
            ("residueInfo", residueInfo, V.Residue_dtype), ("atomInfo", atomInfo, V.Atom_dtype),
            ("grid", grid, np.dtype(np.uint8) if grid_bits else np.dtype(np.float32)),
            ("ff", ff, np.dtype(np.float32)), ("moveArray", moveArray, np.dtype(np.int32))]
    for name, a, dt in spec:
        if not isinstance(a, np.ndarray):
            raise TypeError(f"{name} must be a numpy array")
        if a.dtype != dt:
            raise TypeError(f"{name} has dtype {a.dtype}, expected {dt}")
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError(f"{name} must be C-contiguous")
    info = SimInfo[0]
    need = [("fragmentInfo", fragmentInfo, int(info["fragTypeNum"])),
            ("residueInfo", residueInfo, int(info["totalResNum"])),
            ("atomInfo", atomInfo, int(info["totalAtomNum"])),
            ("grid", grid, grid_bits_size(grid) if grid_bits else 3 * int(info["totalGridNum"])),
            ("ff", ff, 2 * int(info["ffXNum"]) * int(info["ffYNum"])),
            ("moveArray", moveArray, int(info["mcsteps"]))]
    for name, a, n in need:
        if a.size < n:
            raise ValueError(f"{name} holds {a.size} entries, SimInfo requires {n}")


def print_all_info(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray):
    """The state dump printed when SimInfo['showInfo'] > 0 (gcmc/cpp/gcmc.cpp:16-156)."""
    info = SimInfo[0]
    print("\n\nPrinting InfoStruct:\n")
    print(f"Mcsteps: {info['mcsteps']}\nCutoff: {info['cutoff']}\nGrid_dx: {info['grid_dx']}")
    print("Startxyz: (%g, %g, %g)" % tuple(info["startxyz"]))
    print("Cryst: (%g, %g, %g)" % tuple(info["cryst"]))
    print(f"CavityFactor: {info['cavityFactor']}\nFragTypeNum: {info['fragTypeNum']}")
    print(f"TotalGridNum: {info['totalGridNum']}\nTotalResNum: {info['totalResNum']}")
    print(f"TotalAtomNum: {info['totalAtomNum']}")
    print("\n\nPrinting FragmentInfo:\n")
    for i, f in enumerate(fragmentInfo):
        print(f"AtomArray {i + 1}:\nName: {f['name'].decode(errors='replace')}\nMuex: {f['muex']}")
        print(f"Conc: {f['conc']}\nConfBias: {f['confBias']}\nMcTime: {f['mcTime']}\nStartRes: {f['startRes']}")
        print(f"TotalNum: {f['totalNum']}\nMaxNum: {f['maxNum']}\nNum_atoms: {f['num_atoms']}")
        for j in range(f["num_atoms"]):
            a = f["atoms"][j]
            print(f"Atom {j + 1}:\n  Position: ({a['position'][0]:g}, {a['position'][1]:g}, {a['position'][2]:g})"
                  f"\t  Charge: {a['charge']:g}\t  Type: {a['type']}")
        print()
    print("\n\nPrinting Grid:\n")
    for i in range(int(info["totalGridNum"])):
        print(f"Grid {i + 1}: {grid[3 * i]:g}, {grid[3 * i + 1]:g}, {grid[3 * i + 2]:g}")
    print("\n\nPrinting FF:\n")
    X, Y = int(info["ffXNum"]), int(info["ffYNum"])
    for i in range(X):
        for j in range(Y):
            k = i * Y + j
            print(f"FF {i + 1}, {j + 1}:  sigma {ff[2 * k]:g},  epsilon {ff[2 * k + 1]:g}")
    print("\n\nPrinting MoveArray:\n")
    for i in range(int(info["mcsteps"])):
        f, m = divmod(int(moveArray[i]), 4)
        print(f"Move {i + 1}:\tFragType: {fragmentInfo[f]['name'].decode(errors='replace')}\tMoveType: {m}")


def runGCMC(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray, options=None):
    """Run ``mcsteps`` GCMC steps on the GPU, updating the state arrays in place.

    ``options`` (optional, not part of the reference signature) is a
    :class:`pygcmc_b200._native.Options`; the default is the reference's
    semantics (``proposal=0``, ``muex_kcal=0``).  With ``options.grid_bits``
    set, ``grid`` is a gcmc_grid_bits record
    (:func:`pygcmc_b200.system.cavity_bits`) instead of the float list.
    """
    opt = options if options is not None else default_options()
    bits = bool(opt.grid_bits)
    validate_arrays(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray, grid_bits=bits)
    show = int(SimInfo[0]["showInfo"]) > 0 and not bits
    if show:
        print_all_info(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray)
    st = lib().gcmc_run_gcmc(ptr(SimInfo), ptr(fragmentInfo), ptr(residueInfo), ptr(atomInfo), ptr(grid),
                             ptr(ff), ptr(moveArray), __import__("ctypes").byref(opt))
    check(st, "runGCMC")
    if show:
        print_all_info(SimInfo, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray)
    return None


def runGCMC_batch(replicas, options=None):
    """Batched form of :func:`runGCMC` (no counterpart in the reference): every
    replica -- a :class:`pygcmc_b200.system.System` or a 7-tuple of the
    runGCMC arrays -- runs its ``mcsteps`` steps in one device context (one
    pose-energy launch and one accept launch per MC step for all of them; a
    single replica speculates instead, see ``Options.speculate``), and
    each replica's fragmentInfo/residueInfo/atomInfo are updated in place.
    With ``options.grid_bits`` set, each System's ``grid_bits`` record (or a
    tuple's fifth array, a gcmc_grid_bits record) goes in place of the float
    grid."""
    import ctypes
    from ._native import ReplicaIn
    opt = options if options is not None else default_options()
    bits = bool(opt.grid_bits)
    arrays = [r.arrays_for(opt) if hasattr(r, "arrays_for") else tuple(r) for r in replicas]
    for a in arrays:
        validate_arrays(*a, grid_bits=bits)
    arr = (ReplicaIn * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = ReplicaIn(*[ptr(x) for x in a])
    check(lib().gcmc_run_batch(len(arrays), arr, ctypes.byref(opt)), "runGCMC_batch")
    return None
