"""The allocation-free pose-energy entry point (gcmc_energy_poses_noalloc).

Callers that cannot allocate GPU memory where they need trial energies (their
own pool owns the device budget, or their pipeline must not block on
cudaMalloc/cudaFree) pass buffers they already own; this checks, through the C
ABI, that two calls in a row give the energies and group counts of the
allocating entry point gcmc_energy_poses on the same poses -- for a plain and
an Ewald context, with and without residues to skip, on the legacy default
stream and on a stream of the caller's, with and without the group counts --
that a site type outside the pair table is reported at the next sync, and that
requests beyond the fixed scratch are refused.  Kept in its own file, collected
last.
"""
import ctypes

import numpy as np
import pytest

from conftest import energy_close

pytestmark = pytest.mark.gpu


def insertion_poses(oracle, s, ftype, step, n):
    xyz, cen = [], []
    for i in range(n):
        p, c = oracle.insert_pose(s, ftype, step, i)
        xyz.append(p)
        cen.append(c)
    return np.array(xyz, np.float32), np.array(cen, np.float32)


def occupied_poses(s, ftype):
    """The current poses of the type's occupied slots, each skipping its own residue."""
    f = s.fragmentInfo[ftype]
    ns = int(f["num_atoms"])
    xyz, cen, res = [], [], []
    for j in range(int(f["totalNum"])):
        r = int(f["startRes"]) + j
        a0 = int(s.residueInfo[r]["atomStart"])
        xyz.append(s.atomInfo["position"][a0:a0 + ns])
        cen.append(s.residueInfo[r]["position"])
        res.append(r)
    return np.array(xyz, np.float32), np.array(cen, np.float32), np.array(res, np.int32)


def call_noalloc(L, eng, xyz, q, ty, cen, self_res, stream_handle, want_groups):
    import torch
    dev = torch.device("cuda:0")
    n, ns = xyz.shape[0], xyz.shape[1]
    d_xyz = torch.from_numpy(xyz).to(dev)
    d_q = torch.from_numpy(q).to(dev)
    d_t = torch.from_numpy(ty).to(dev)
    d_c = torch.from_numpy(cen).to(dev)
    d_self = None if self_res is None else torch.from_numpy(self_res).to(dev)
    d_out = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    d_ng = torch.full((n,), -1, dtype=torch.int32, device=dev) if want_groups else None
    torch.cuda.synchronize()  # the inputs are in place before a launch on another stream
    st = L.gcmc_energy_poses_noalloc(eng.handle, 0, d_xyz.data_ptr(), d_q.data_ptr(), d_t.data_ptr(), ns,
                                     d_c.data_ptr(), None if d_self is None else d_self.data_ptr(), n,
                                     d_out.data_ptr(), None if d_ng is None else d_ng.data_ptr(),
                                     ctypes.c_void_p(stream_handle))
    assert st == 0
    torch.cuda.synchronize()
    eng.sync()
    return d_out.cpu().numpy(), (None if d_ng is None else d_ng.cpu().numpy())


@pytest.mark.parametrize("case", ["plain", "self_slots", "own_stream", "no_group_counts", "ewald"])
def test_noalloc_matches_allocating_entry_point(oracle_lib, protein_small, case):
    import torch
    from pygcmc_b200._native import default_options, lib
    from pygcmc_b200.engine import Engine

    s = protein_small
    L = lib()
    opts = default_options()
    if case == "ewald":
        opts = default_options(pme=1, pme_alpha=0.32)
        for a in range(3):
            opts.pme_grid[a] = 48
    side = torch.cuda.Stream() if case == "own_stream" else None
    handle = side.cuda_stream if side is not None else 1  # 1: cudaStreamLegacy
    with Engine(s.copy(), opts) as eng:
        for call, (ftype, step, n) in enumerate([(0, 7, 300), (1, 9, 37)]):  # the second call is smaller
            f = s.fragmentInfo[ftype]
            ns = int(f["num_atoms"])
            q = f["atoms"]["charge"][:ns].copy()
            ty = f["atoms"]["type"][:ns].astype(np.int32)
            if case == "self_slots":
                xyz, cen, self_res = occupied_poses(s, ftype)
                assert len(self_res) > 0
            else:
                xyz, cen = insertion_poses(oracle_lib, s, ftype, step, n)
                self_res = None
            e_ref, ng_ref = eng.energy_poses(xyz, q, ty, cen, self_res)
            e, ng = call_noalloc(L, eng, xyz, q, ty, cen, self_res, handle, case != "no_group_counts")
            if ng is not None:
                assert np.array_equal(ng, ng_ref), (case, call)
            assert energy_close(e, e_ref).all(), (case, call, np.abs(e - e_ref).max())


def test_noalloc_reports_bad_site_type(oracle_lib, protein_small):
    from pygcmc_b200._native import GcmcError, lib
    from pygcmc_b200.engine import Engine
    s = protein_small
    L = lib()
    ffx = int(s.SimInfo[0]["ffXNum"])
    f = s.fragmentInfo[0]
    ns = int(f["num_atoms"])
    q = f["atoms"]["charge"][:ns].copy()
    ty = f["atoms"]["type"][:ns].astype(np.int32)
    ty[ns - 1] = ffx  # one row past the pair table
    xyz, cen = insertion_poses(oracle_lib, s, 0, 3, 16)
    with Engine(s.copy()) as eng:
        with pytest.raises(GcmcError):
            call_noalloc(L, eng, xyz, q, ty, cen, None, 1, True)
        assert eng.device_error() & 16


def test_noalloc_refuses_oversized_requests(protein_small):
    from pygcmc_b200._native import lib
    from pygcmc_b200.engine import Engine
    L = lib()
    with Engine(protein_small.copy()) as eng:
        fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
        st = L.gcmc_energy_poses_noalloc(eng.handle, 0, fake, fake, fake, 4, fake, None, 1_000_000, fake, None,
                                         None)
        assert st == 3
