"""A small, fixed GCMC run for kernel profiling (ncu) and per-kernel timing.

    python -m pygcmc_b200.profile_case [--warm 64] [--steps 24] [--system protein|water|batched]

Builds the synthetic protein system (6000 fixed atoms, 64 A box, 8 fragments,
confBias 1000; `batched`: 64 replicas of 2000-40000 atoms in one context),
advances it `--warm` steps through the graph-captured step loop, then launches
`--steps` steps kernel by kernel with CUDA events around each launch and
prints the per-step kernel times.  Under ncu, the k_energy and k_accept
launches after the first `--warm` are the individually launched ones.
"""
import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--warm", type=int, default=64)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--system", choices=["protein", "water", "batched"], default="protein")
    ap.add_argument("--cells", type=int, default=2)
    ap.add_argument("--split", type=int, default=0, help="work items per step (0: default)")
    ap.add_argument("--variant", type=int, default=0, help="pose-energy register budget variant")
    a = ap.parse_args()
    from . import system as S
    from ._native import default_options
    from .engine import Engine
    total = a.warm + a.steps + 64
    if a.system == "protein":
        s = S.protein_system(seed=1, mcsteps=total)
    elif a.system == "water":
        s = S.water_box(seed=1, mcsteps=total)
    else:
        s = S.replica_batch(n_rep=64, seed=1, mcsteps=total)
    opt = default_options(cells_per_cutoff=a.cells, energy_variant=a.variant)
    if a.split > 0:
        opt.split_items = a.split
    with Engine(s, opt) as eng:
        eng.run(a.warm)
        eng.sync()
        te, ta, mv = eng.run_profiled(a.steps)
        print(json.dumps({"move": (mv % 4).tolist(), "energy_us": [round(float(x) * 1e3, 2) for x in te],
                          "accept_us": [round(float(x) * 1e3, 2) for x in ta], "counters": eng.counters()}))


if __name__ == "__main__":
    main()
