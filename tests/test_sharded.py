"""Auxiliary-shell sharding of one molecule over ranks (CPU: gloo, world size 2).

The partition and the all-gather of the raw contraction are the product's
(pysisyphus_addons.diabatization.sharded); the per-rank compute is injected:
here the oracle's raw contraction of each rank's sub-basis and a LAPACK solve,
so the test runs without a GPU. The gathered raw contraction must equal the
oracle's full one bit for bit (the oracle computes every auxiliary shell's
rows independently of the others), and df and the tensor must match the
oracle's single-process results."""

import os
import socket

import numpy as np
import pytest
import scipy.linalg as sl

import oracle
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.diabatization import sharded as sh


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.exponential(size=101)
    for nr in (1, 2, 3, 8):
        ranges = sh.partition_aux_shells(costs, nr)
        assert len(ranges) == nr and ranges[0][0] == 0 and ranges[-1][1] == len(costs)
        assert all(a <= b for a, b in ranges)
        assert all(ranges[i][1] == ranges[i + 1][0] for i in range(nr - 1))
        loads = [costs[a:b].sum() for a, b in ranges]
        # a prefix split is within one shell's cost of the even share
        assert max(loads) <= costs.sum() / nr + costs.max() + 1e-12


def test_partition_edge_cases():
    assert sh.partition_aux_shells([], 3) == [(0, 0), (0, 0), (0, 0)]
    assert sh.partition_aux_shells([5.0], 2) in ([(0, 1), (1, 1)], [(0, 0), (0, 1)])
    r = sh.partition_aux_shells(np.zeros(6), 3)
    assert r[0][0] == 0 and r[-1][1] == 6
    with pytest.raises(ValueError):
        sh.partition_aux_shells([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = config_workload("cfg1")
        oracle.set_boys_mode("reference")
        costs = sh.aux_shell_costs(w.shells, w.shells_aux, oracle.int_schwarz_bra(w.shells),
                                   oracle.int_schwarz_aux(w.shells_aux), len(w.densities))
        seen = {}

        def raw_fn(shells, sub, D):
            oracle.set_skip_metric(1)
            try:
                raw = oracle.contract_coulomb_densities_2d(shells, sub, D) if len(sub) else np.zeros((0, len(D)))
            finally:
                oracle.set_skip_metric(0)
            return torch.from_numpy(np.ascontiguousarray(raw.T))

        def solve_fn(shells_aux, raw_full, nstates):
            raw = raw_full.numpy().T  # (naux, nd)
            seen["raw"] = raw.copy()
            M = oracle.int2c2e(shells_aux)
            df = sl.solve_triangular(sl.cholesky(M, lower=True), raw, lower=True)
            R = oracle.coulomb_from_df(df, nstates)
            return np.ascontiguousarray(df.T), R.ravel(order="F")

        df, R, rng = sh.contract_coulomb_densities_4d_sharded(w.shells, w.shells_aux, w.densities, raw_fn=raw_fn,
                                                              solve_fn=solve_fn, costs=costs)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), df=df, R=R, raw=seen["raw"], lo=rng[0], hi=rng[1])
    finally:
        dist.destroy_process_group()


def test_sharded_world2_matches_single_process(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    w = config_workload("cfg1")
    oracle.set_boys_mode("reference")
    oracle.set_skip_metric(1)
    try:
        raw_ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        oracle.set_skip_metric(0)
    df_ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    R_ref = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    # the two ranks own consecutive, non-empty ranges covering every shell
    assert int(res[0]["lo"]) == 0 and int(res[0]["hi"]) == int(res[1]["lo"])
    assert int(res[1]["hi"]) == len(w.shells_aux) and 0 < int(res[0]["hi"]) < len(w.shells_aux)
    for r in res:
        np.testing.assert_array_equal(r["raw"], raw_ref)  # gathered rows are the full contraction
        # LAPACK dtrsm here, dtrtri + dtrmm in the oracle driver: 3e-11 as in the GPU tests
        np.testing.assert_allclose(r["df"], df_ref, atol=3e-11, rtol=0)
        np.testing.assert_allclose(r["R"], R_ref, atol=1e-12 + 1e-13 * np.abs(R_ref).max(), rtol=0)
    np.testing.assert_array_equal(res[0]["R"], res[1]["R"])
