"""Golden pose energies from the reference's own calcEnergy kernel.

    python tests/golden/make_ref_energies.py OUT.npz      (needs a CUDA GPU)

Loads oracle/_ref/libref_energy.so -- a 128-thread-per-pose probe kernel that
calls pyGCMC's calcEnergy (gcmc/cpp/gcmc_energy.h:142-204) compiled unmodified
from the reference header by `make -C oracle ref` -- and evaluates seeded poses
(insertion poses of every fragment type and the current poses of occupied
slots, with self exclusion) on two small synthetic systems.  The output holds
the systems' state arrays, the poses and the reference kernel's FP32 energies;
tests/test_ref_golden.py checks the CPU oracle against it.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def poses_for(oracle, s, per_type=48):
    from pygcmc_b200 import values as V
    out = []
    for t, f in enumerate(s.fragmentInfo):
        ns = int(f["num_atoms"])
        rows = []
        for i in range(per_type):
            xyz, c = oracle.insert_pose(s, t, 3, i)
            rows.append((xyz, c, -1))
        for j in range(min(int(f["totalNum"]), per_type)):
            r = s.residueInfo[int(f["startRes"]) + j]
            a0 = int(r["atomStart"])
            rows.append((s.atomInfo["position"][a0:a0 + ns].copy(), r["position"].copy(), int(f["startRes"]) + j))
        arr = np.zeros(len(rows), dtype=V.AtomArray_dtype)
        for p, (xyz, c, self_res) in enumerate(rows):
            arr[p]["num_atoms"] = ns
            arr[p]["startRes"] = self_res
            arr[p]["atoms"]["position"][:ns] = xyz
            arr[p]["atoms"]["charge"][:ns] = f["atoms"]["charge"][:ns]
            arr[p]["atoms"]["type"][:ns] = f["atoms"]["type"][:ns]
        cen = np.array([c for _, c, _ in rows], np.float32)
        out.append((t, arr, cen))
    return out


def main(path):
    import oracle
    from pygcmc_b200 import system as S
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_energy.so"))
    L.ref_probe_energies.restype = ctypes.c_int
    L.ref_probe_energies.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_int, ctypes.c_void_p]
    systems = {
        "protein": S.protein_system(seed=11, n_atoms=2500, box=48.0, radius=16.0, mcsteps=64, conf_bias=64),
        "water": S.water_box(n_water=300, box=30.0, seed=12, mcsteps=64, conf_bias=64),
    }
    data = {}
    for name, s in systems.items():
        for k, a in zip(("SimInfo", "fragmentInfo", "residueInfo", "atomInfo", "ff"),
                        (s.SimInfo, s.fragmentInfo, s.residueInfo, s.atomInfo, s.ff)):
            data[f"{name}_{k}"] = a
        poses, cens, ts, es = [], [], [], []
        for t, arr, cen in poses_for(oracle, s):
            out = np.zeros(len(arr), np.float32)
            rc = L.ref_probe_energies(s.SimInfo.ctypes.data, s.fragmentInfo.ctypes.data, s.residueInfo.ctypes.data,
                                      s.atomInfo.ctypes.data, s.ff.ctypes.data, arr.ctypes.data, cen.ctypes.data,
                                      len(arr), out.ctypes.data)
            if rc != 0:
                raise RuntimeError(f"reference probe failed ({rc})")
            poses.append(arr)
            cens.append(cen)
            ts.append(np.full(len(arr), t, np.int32))
            es.append(out)
        data[f"{name}_poses"] = np.concatenate(poses)
        data[f"{name}_centres"] = np.concatenate(cens)
        data[f"{name}_ptype"] = np.concatenate(ts)
        data[f"{name}_ref_energy"] = np.concatenate(es)
    np.savez_compressed(path, **data)
    print(f"wrote {path}: " + ", ".join(f"{n}: {len(data[n + '_ref_energy'])} poses" for n in systems))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                           "ref_kernel_energies.npz"))
