"""The cavity grid as a voxel bit set (gcmc_options.grid_bits = 1): the engine
expands the gcmc_grid_bits record on the device into the insertion base
points; the chains must equal those run from the reference's float list
(needs a B200).

* Engine runs (one replica, a batch) from the bit set are bit-identical to
  runs from the float list: per-step logs, logged pose energies, counters,
  final state.
* The batched and single drop-in calls with bit sets update the caller's
  arrays exactly as with float lists.
* Bits past the last voxel are ignored.
* A record whose marked voxels do not number totalGridNum is refused with
  GCMC_ERR_ARG (the device counts them and writes no point past the
  buffer).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LOG_KMAX = 1024


def _run(systems, nsteps, **opt):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, **opt)
    with Engine([s.copy() for s in systems], opts) as eng:
        eng.run(nsteps)
        eng.sync()
        assert eng.device_error() == 0
        out = []
        for r in range(len(systems)):
            logs, E = eng.logs(r)
            out.append((logs, E, eng.download(r), eng.counters(r)))
    return out


def _same(a, b):
    for (la, Ea, fa, ca), (lb, Eb, fb, cb) in zip(a, b):
        for f in la.dtype.names:
            assert np.array_equal(la[f], lb[f]), f
        assert np.array_equal(Ea.view(np.uint64), Eb.view(np.uint64))
        assert ca == cb
        assert np.array_equal(fa.fragmentInfo["totalNum"], fb.fragmentInfo["totalNum"])
        assert np.array_equal(fa.atomInfo.view(np.uint8), fb.atomInfo.view(np.uint8))
        assert np.array_equal(fa.residueInfo.view(np.uint8), fb.residueInfo.view(np.uint8))


def _inserted(out):
    return sum(int(((lg["move"] == 0) & (lg["n_accept"] > 0)).sum()) for lg, _, _, _ in out)


@pytest.mark.parametrize("which", ["protein", "water"])
def test_bit_set_equals_float_list(request, which):
    sysm = request.getfixturevalue(f"{which}_small")
    n = 120
    ref = _run([sysm], n)
    bits = _run([sysm], n, grid_bits=1)
    _same(ref, bits)
    assert _inserted(bits) > 0


def test_bit_set_batch(protein_small, water_small):
    batch = [protein_small, water_small, protein_small]
    n = 80
    _same(_run(batch, n), _run(batch, n, grid_bits=1))


def test_drop_in_calls_with_bit_sets(protein_small, water_small):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.gpu import runGCMC, runGCMC_batch
    nsteps = 60
    a = [s.copy() for s in (protein_small, water_small)]
    b = [s.copy() for s in (protein_small, water_small)]
    for s in a + b:
        s.SimInfo[0]["mcsteps"] = nsteps
    runGCMC_batch(a, default_options())
    runGCMC_batch(b, default_options(grid_bits=1))
    for x, y in zip(a, b):
        for f in ("fragmentInfo", "residueInfo", "atomInfo"):
            assert np.array_equal(getattr(x, f).view(np.uint8), getattr(y, f).view(np.uint8)), f
    c, d = protein_small.copy(), protein_small.copy()
    for s in (c, d):
        s.SimInfo[0]["mcsteps"] = nsteps
    runGCMC(*c.arrays())
    runGCMC(*d.arrays_for(default_options(grid_bits=1)), options=default_options(grid_bits=1))
    for f in ("fragmentInfo", "residueInfo", "atomInfo"):
        assert np.array_equal(getattr(c, f).view(np.uint8), getattr(d, f).view(np.uint8)), f


def test_bits_past_the_last_voxel_are_ignored(water_small):
    s = water_small.copy()
    rec = s.grid_bits
    n = np.frombuffer(rec[32:44].tobytes(), np.int32).astype(np.int64)
    nvox = int(n.prod())
    words = rec[48:].view(np.uint32)
    if nvox % 32 == 0:
        pytest.skip("the voxel count fills its last word")
    words[-1] |= np.uint32(0xFFFFFFFF) << np.uint32(nvox % 32)
    _same(_run([water_small], 60, grid_bits=1), _run([s], 60, grid_bits=1))


def test_no_grid_array_without_insertions(protein_small):
    """A schedule without insertions needs no cavity grid: a NULL grid argument (either
    grid form) runs the same chain as with the grid."""
    import ctypes
    from pygcmc_b200._native import ReplicaIn, check, default_options, lib, ptr
    from pygcmc_b200.engine import Engine
    n = 60
    s = protein_small.copy()
    mv = s.moveArray.copy()
    mv[(mv % 4) == 0] += 1  # insertions become deletions
    s.moveArray = mv
    ref = _run([s], n)
    for bits in (0, 1):
        t = s.copy()
        opts = default_options(log_steps=n, log_kmax=LOG_KMAX, grid_bits=bits)
        arr = (ReplicaIn * 1)()
        a = t.arrays()
        arr[0] = ReplicaIn(*[ptr(x) for x in a[:4]], None, *[ptr(x) for x in a[5:]])
        h = ctypes.c_void_p()
        check(lib().gcmc_create(1, arr, ctypes.byref(opts), None, ctypes.byref(h)), "gcmc_create")
        eng = Engine.__new__(Engine)
        eng.systems, eng.options, eng._in, eng._h = [t], opts, arr, h
        with eng:
            eng.run(n)
            eng.sync()
            assert eng.device_error() == 0
            logs, E = eng.logs(0)
            out = [(logs, E, eng.download(0), eng.counters(0))]
        _same(ref, out)


def test_count_mismatch_is_refused(protein_small):
    from pygcmc_b200._native import GcmcError, default_options
    from pygcmc_b200.engine import Engine
    s = protein_small.copy()
    s.SimInfo[0]["totalGridNum"] = int(s.SimInfo[0]["totalGridNum"]) - 1
    with pytest.raises(GcmcError) as e:
        Engine([s], default_options(grid_bits=1))
    assert e.value.status == 2
