"""The multi-process ("replicas only") path on the CPU: two gloo ranks, each
advancing its own replica (seed by rank) with the oracle, with the host-side
collectives bench.py uses (barrier, max / sum over ranks).  Each rank's chain
must equal the same replica run alone in one process."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _chain(seed, nsteps=12):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from pygcmc_b200 import system as S
    s = S.water_box(n_water=80, box=16.0, seed=seed, mcsteps=nsteps, conf_bias=16)
    logs, _ = oracle.run(s, nsteps, opts=oracle.options(), kmax=64, threads=1)
    return {"totalNum": s.fragmentInfo["totalNum"].tolist(), "accepts": logs["n_accept"].tolist()}


def _rank(rank, ws, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from pygcmc_b200 import replicas
    assert replicas.env() == (ws, rank, rank)
    replicas.init("gloo", timeout_s=60)
    try:
        replicas.barrier(ws)
        res = _chain(replicas.replica_seed(5, rank, 3))
        slowest = replicas.max_over_ranks(float(rank + 1), ws)
        total = replicas.sum_over_ranks(float(sum(res["accepts"])), ws)
        replicas.barrier(ws)
        res.update({"max": slowest, "sum": total})
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        replicas.finalize()


def test_two_gloo_ranks_run_independent_replicas(oracle_lib, tmp_path):
    ws = 2
    port = _free_port()
    mp.start_processes(_rank, args=(ws, port, str(tmp_path)), nprocs=ws, join=True, start_method="spawn")
    results = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]
    assert all(r["max"] == float(ws) for r in results)
    assert results[0]["sum"] == results[1]["sum"] == float(sum(sum(r["accepts"]) for r in results))
    for r in range(ws):
        solo = _chain(5 + 3 * r)
        assert results[r]["totalNum"] == solo["totalNum"] and results[r]["accepts"] == solo["accepts"]
