"""The CPU oracle against energies computed by the reference's own CUDA
calcEnergy (fixture made on a B200 by tests/golden/make_ref_energies.py from
the unmodified reference header).  No GPU needed."""
import os

import numpy as np
import pytest

from conftest import ROOT, energy_close

FIX = os.path.join(ROOT, "tests", "golden", "ref_kernel_energies.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(FIX), reason="reference-kernel fixture not generated")


def load(name):
    from pygcmc_b200.system import System
    d = np.load(FIX)
    s = System(d[f"{name}_SimInfo"], d[f"{name}_fragmentInfo"], d[f"{name}_residueInfo"], d[f"{name}_atomInfo"],
               np.zeros(3, np.float32), d[f"{name}_ff"], np.zeros(0, np.int32))
    return s, d[f"{name}_poses"], d[f"{name}_centres"], d[f"{name}_ptype"], d[f"{name}_ref_energy"]


@pytest.mark.parametrize("name", ["protein", "water"])
def test_oracle_matches_reference_kernel(oracle_lib, name):
    s, poses, cens, ptype, e_ref = load(name)
    worst_mirror, worst64 = 0.0, 0.0
    for t in np.unique(ptype):
        sel = np.flatnonzero(ptype == t)
        ns = int(poses[sel[0]]["num_atoms"])
        xyz = np.ascontiguousarray(poses["atoms"]["position"][sel, :ns])
        q = poses["atoms"]["charge"][sel[0], :ns]
        ty = poses["atoms"]["type"][sel[0], :ns]
        self_res = poses["startRes"][sel].astype(np.int32)
        e32, ng32, _ = oracle_lib.energy_batch(s, xyz, q, ty, cens[sel], self_res, mode=1)
        e64, ng64, _, l1 = oracle_lib.energy_batch(s, xyz, q, ty, cens[sel], self_res, mode=0, want_l1=True)
        ref = e_ref[sel].astype(np.float64)
        assert np.array_equal(ng32, ng64)
        # errors are bounded relative to l1 = sum of |pair terms| (the sum's
        # condition): the reference kernel's own FP32 summation differs from
        # the FP64 restatement by a few 1e-6 of l1, and the FP32 mirror of its
        # arithmetic (up to pow() and fused multiply-add choices) likewise
        d32 = np.abs(e32 - ref) / np.maximum(l1, 1e-30)
        d64 = np.abs(e64 - ref) / np.maximum(l1, 1e-30)
        worst_mirror = max(worst_mirror, float(d32.max()))
        worst64 = max(worst64, float(d64.max()))
        assert (np.abs(e32 - ref) <= np.maximum(2e-5 * l1, 1e-6)).all(), (t, d32.max())
        assert (np.abs(e64 - ref) <= np.maximum(2e-5 * l1, 1e-6)).all(), (t, d64.max())
    print(f"{name}: |mirror - reference| / l1 <= {worst_mirror:.2e}; |FP64 - reference| / l1 <= {worst64:.2e}")
