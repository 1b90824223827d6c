"""The allocation-free pose-energy entry point (gcmc_energy_poses_noalloc).

Callers that cannot allocate GPU memory where they need trial energies (their
own pool owns the device budget, or their pipeline must not block on
cudaMalloc/cudaFree) pass buffers they already own; this checks, through the C
ABI, that two calls in a row give the energies and group counts of the
allocating entry point gcmc_energy_poses on the same poses, and that requests
beyond the fixed scratch are refused.  Kept in its own file, collected last.
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


def test_noalloc_matches_allocating_entry_point(oracle_lib, protein_small):
    import torch
    from pygcmc_b200._native import lib
    from pygcmc_b200.engine import Engine

    s = protein_small
    L = lib()
    with Engine(s.copy()) as eng:
        for call, (ftype, step, n) in enumerate([(0, 7, 300), (1, 9, 37)]):  # the second call is smaller
            f = s.fragmentInfo[ftype]
            ns = int(f["num_atoms"])
            q = f["atoms"]["charge"][:ns].copy()
            ty = f["atoms"]["type"][:ns].astype(np.int32)
            xyz, cen = insertion_poses(oracle_lib, s, ftype, step, n)
            e_ref, ng_ref = eng.energy_poses(xyz, q, ty, cen)

            dev = torch.device("cuda:0")
            d_xyz = torch.from_numpy(xyz).to(dev)
            d_q = torch.from_numpy(q).to(dev)
            d_t = torch.from_numpy(ty).to(dev)
            d_c = torch.from_numpy(cen).to(dev)
            d_out = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            d_ng = torch.full((n,), -1, dtype=torch.int32, device=dev)
            stream = torch.cuda.current_stream()
            st = L.gcmc_energy_poses_noalloc(eng.handle, 0, d_xyz.data_ptr(), d_q.data_ptr(), d_t.data_ptr(), ns,
                                             d_c.data_ptr(), None, n, d_out.data_ptr(), d_ng.data_ptr(),
                                             ctypes.c_void_p(stream.cuda_stream or 1))  # 1: cudaStreamLegacy
            assert st == 0
            torch.cuda.synchronize()
            eng.sync()
            e = d_out.cpu().numpy()
            ng = d_ng.cpu().numpy()
            assert np.array_equal(ng, ng_ref), call
            assert energy_close(e, e_ref).all(), (call, np.abs(e - e_ref).max())


def test_noalloc_refuses_oversized_requests(protein_small):
    from pygcmc_b200._native import lib
    from pygcmc_b200.engine import Engine
    L = lib()
    with Engine(protein_small.copy()) as eng:
        fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
        st = L.gcmc_energy_poses_noalloc(eng.handle, 0, fake, fake, fake, 4, fake, None, 1_000_000, fake, None,
                                         None)
        assert st == 3
