"""The drop-in boundary as the reference's users reach it (needs a B200).

* the reference's own CPython binding (gcmc/cpp/gcmc.cpp:159-224, compiled
  unmodified as setup.py:92-128 compiles it, but linked to this library's
  runGCMC_cuda instead of the reference's gcmc.o; built into oracle/_ref/binding
  by `make -C oracle ref`) runs a trajectory whose results equal an Engine run
  of the same steps, in place in the caller's numpy arrays and returning None,
  as gcmc/python/gcmc.py:41-49 calls it;
* the `void runGCMC_cuda` export called through ctypes, followed by
  gcmc_last_status(): 0 and the Engine's results on good input, GCMC_ERR_ARG
  and untouched arrays on inconsistent input.
"""
import ctypes
import glob
import importlib.util
import os

import numpy as np
import pytest

from conftest import ROOT
from test_gpu_parity import engine_trajectory, occupied_atoms, occupied_res

pytestmark = pytest.mark.gpu


def reference_binding():
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", "binding", "gpu*.so"))
    if not paths:
        pytest.skip("the reference's binding was not built (make -C oracle ref needs the pyGCMC sources)")
    spec = importlib.util.spec_from_file_location("gpu", paths[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def assert_same_state(a, b):
    assert np.array_equal(a.fragmentInfo["totalNum"], b.fragmentInfo["totalNum"])
    at = occupied_atoms(b)
    assert np.array_equal(a.atomInfo["position"][at], b.atomInfo["position"][at])
    r = occupied_res(b)
    assert np.array_equal(a.residueInfo["position"][r], b.residueInfo["position"][r])


@pytest.mark.parametrize("which", ["protein_small", "water_small"])
def test_reference_binding_drives_the_engine(request, which):
    gpu = reference_binding()
    system = request.getfixturevalue(which)
    s = system.copy()
    n = int(s.SimInfo[0]["mcsteps"])
    # the call of gcmc/python/gcmc.py:41-49
    assert gpu.runGCMC(s.SimInfo, s.fragmentInfo, s.residueInfo, s.atomInfo, s.grid, s.ff, s.moveArray) is None
    _, _, final, _ = engine_trajectory(system, n)
    assert_same_state(s, final)
    assert (s.fragmentInfo["totalNum"] != system.fragmentInfo["totalNum"]).any()  # the run moved something


def test_runGCMC_cuda_export_and_last_status(protein_small):
    from pygcmc_b200._native import lib
    L = lib()
    fn = L.runGCMC_cuda
    fn.restype = None
    fn.argtypes = [ctypes.c_void_p] * 7
    s = protein_small.copy()
    n = int(s.SimInfo[0]["mcsteps"])
    fn(*[a.ctypes.data for a in s.arrays()])
    assert L.gcmc_last_status() == 0
    _, _, final, _ = engine_trajectory(protein_small, n)
    assert_same_state(s, final)
    # inconsistent input: a move of a fragment type that does not exist
    bad = protein_small.copy()
    bad.moveArray[5] = 4 * len(bad.fragmentInfo)
    before = bad.copy()
    fn(*[a.ctypes.data for a in bad.arrays()])
    assert L.gcmc_last_status() == 2  # GCMC_ERR_ARG
    assert np.array_equal(bad.atomInfo, before.atomInfo)
    assert np.array_equal(bad.fragmentInfo, before.fragmentInfo)
    # the next good call succeeds again
    s2 = protein_small.copy()
    fn(*[a.ctypes.data for a in s2.arrays()])
    assert L.gcmc_last_status() == 0
    assert_same_state(s2, final)
