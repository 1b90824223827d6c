"""C ABI: struct layouts, exported symbols and argument checks (no GPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gcmc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "return")))


def test_numpy_dtypes_match_reference_sizes():
    from pygcmc_b200 import values as V
    assert (V.Atom_dtype.itemsize, V.AtomArray_dtype.itemsize, V.Info_dtype.itemsize,
            V.Residue_dtype.itemsize) == (20, 436, 76, 20)


def test_c_struct_sizes(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "gcmc_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(Atom), sizeof(AtomArray),'
                   ' sizeof(InfoStruct), sizeof(residue), sizeof(gcmc_options), sizeof(gcmc_step_log),'
                   ' offsetof(AtomArray, atoms));printf("%zu %zu\\n", sizeof(gcmc_grid_bits),'
                   ' offsetof(gcmc_grid_bits, n));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    out = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    from pygcmc_b200._native import Options
    from pygcmc_b200.values import StepLog_dtype, AtomArray_dtype
    assert out[:4] == [20, 436, 76, 20]
    assert out[4] == ctypes.sizeof(Options)
    assert out[5] == StepLog_dtype.itemsize
    assert out[6] == AtomArray_dtype.fields["atoms"][1]
    from pygcmc_b200.gpu import GRID_BITS_HEADER
    assert out[7:9] == [GRID_BITS_HEADER, 32]


def test_library_exports_every_declared_symbol(native_lib):
    names = declared_functions()
    assert "runGCMC_cuda" in names and "gcmc_energy_poses" in names
    missing = [n for n in names if not hasattr(native_lib, n)]
    assert not missing, missing


def test_status_strings_and_defaults(native_lib):
    from pygcmc_b200._native import default_options
    assert native_lib.gcmc_status_string(0) == b"ok"
    o = default_options()
    assert o.proposal == 0 and o.muex_kcal == 0 and o.cells_per_cutoff == 2


def test_runGCMC_rejects_bad_arrays(water_small):
    from pygcmc_b200.gpu import runGCMC
    s = water_small.copy()
    with pytest.raises(TypeError):
        runGCMC(s.SimInfo, s.fragmentInfo, s.residueInfo, s.atomInfo, s.grid.astype(np.float64), s.ff, s.moveArray)
    with pytest.raises(ValueError):
        runGCMC(s.SimInfo, s.fragmentInfo, s.residueInfo[:5], s.atomInfo, s.grid, s.ff, s.moveArray)


def test_create_rejects_inconsistent_input_without_gpu(water_small):
    """Argument validation runs before any device call, so it is testable here."""
    from pygcmc_b200._native import GcmcError
    from pygcmc_b200.engine import Engine
    s = water_small.copy()
    s.moveArray[3] = 4 * 7  # fragment type 7 does not exist
    with pytest.raises(GcmcError) as e:
        Engine(s)
    assert e.value.status == 2
    s = water_small.copy()
    s.fragmentInfo[0]["confBias"] = 5000
    with pytest.raises(GcmcError) as e:
        Engine(s)
    assert e.value.status == 3


def test_batched_create_validates_every_replica_without_gpu(water_small, protein_small):
    """A batch's replicas are validated on host threads before any device call: a
    bad replica anywhere in the batch is reported (status 2), a good batch gets
    past validation (status 5 = no CUDA device here, or 0 on a GPU box)."""
    from pygcmc_b200._native import GcmcError
    from pygcmc_b200.engine import Engine
    good = [water_small.copy() if i % 2 else protein_small.copy() for i in range(6)]
    for bad_at in (0, 3, 5):
        batch = [s.copy() for s in good]
        atoms = batch[bad_at].atomInfo
        atoms["type"][0] = 999  # a fixed (or occupied) atom's type outside the pair table
        with pytest.raises(GcmcError) as e:
            Engine(batch)
        assert e.value.status == 2
    try:
        Engine([s.copy() for s in good]).close()
    except GcmcError as e:
        assert e.status == 5


def test_reference_binding_links_to_this_library():
    """The reference's CPython binding (gcmc/cpp/gcmc.cpp, unmodified) built
    against libgcmc_b200.so loads and exposes runGCMC (calling it needs a GPU)."""
    import glob
    import importlib.util
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", "binding", "gpu*.so"))
    if not paths:
        pytest.skip("the reference's binding was not built (make -C oracle ref needs the pyGCMC sources)")
    out = subprocess.check_output(["ldd", paths[0]]).decode()
    assert "libgcmc_b200.so" in out and "not found" not in out
    spec = importlib.util.spec_from_file_location("gpu", paths[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert callable(mod.runGCMC)
