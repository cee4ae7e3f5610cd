"""The device side of the auxiliary-shell sharding on one GPU.

Each rank's part -- the raw contraction of a consecutive range of auxiliary
shells (pa_df_2d with the metric skipped, on the sub-basis) -- is run for
every range of a 3-way partition in turn, the parts are concatenated as the
all-gather would, and pa_df_solve produces df and the tensor. They must
match the single-call path (pa_df_4d): the raw rows at 1e-14 of their largest
element (a sub-basis changes the work-item split and so the summation order
of the bra chunks), df and the tensor at the tolerances of the other
single-molecule tests. A one-rank process group runs the full
contract_coulomb_densities_4d_sharded through its gather."""

import os
import socket

import numpy as np
import pytest

from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.shells import Shells
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.diabatization import intor as dia
from pysisyphus_addons.diabatization import sharded as sh
from pysisyphus_addons.intor import intor as sch

pytestmark = pytest.mark.gpu


def close(x, ref, rel_of_max, atol=0.0):
    tol = atol + rel_of_max * np.abs(ref).max()
    err = np.abs(x - ref).max()
    assert err <= tol, f"max abs err {err:.3e} > {tol:.3e}"


@pytest.mark.parametrize("key", ["cfg1", "cfg2"])
def test_shards_then_solve_match_single_call(key):
    import torch

    torch.cuda.set_device(0)
    nat.set_boys_mode("reference")
    w = config_workload(key)
    nd = len(w.densities)
    costs = sh.aux_shell_costs(w.shells, w.shells_aux, sch.int_schwarz_bra(w.shells),
                               sch.int_schwarz_aux(w.shells_aux), nd)
    ranges = sh.partition_aux_shells(costs, 3)
    loads = [costs[a:b].sum() for a, b in ranges]
    assert max(loads) <= costs.sum() / 3 + costs.max()
    dens = torch.from_numpy(np.ascontiguousarray(w.densities)).cuda()
    parts = [sh.raw_contraction_device(w.shells, Shells(w.shells_aux.shells[a:b]), dens) for a, b in ranges]
    raw = torch.cat(parts, dim=1).contiguous()
    nat.set_skip_metric(1)
    try:
        raw_ref = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        nat.set_skip_metric(0)
    close(raw.cpu().numpy().T, raw_ref, 1e-14)
    df, R = sh.solve_device(w.shells_aux, raw, w.nstates)
    df_ref = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    R_ref = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    # same raw input up to summation order: the solve amplifies it by the metric's conditioning
    tol_df, tol_R = (3e-11, 1e-12) if key == "cfg1" else (1e-6, 5e-9)
    close(df.cpu().numpy().T, df_ref, 0.0, atol=tol_df)
    close(R.cpu().numpy().reshape((w.nstates,) * 4, order="F"), R_ref, tol_R, atol=1e-12)
    # the solve of the single call's own raw contraction is that call's df, bit for bit
    df2, R2 = sh.solve_device(w.shells_aux, torch.from_numpy(np.ascontiguousarray(raw_ref.T)).cuda(), w.nstates)
    np.testing.assert_array_equal(df2.cpu().numpy().T, df_ref)
    np.testing.assert_array_equal(R2.cpu().numpy().reshape((w.nstates,) * 4, order="F"), R_ref)


def test_one_rank_group_runs_the_device_parts():
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    nat.set_boys_mode("reference")
    w = config_workload("cfg1")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        # gloo gathers host tensors: the device parts go through the host
        def raw_fn(shells, sub, D):
            return sh.raw_contraction_device(shells, sub, torch.from_numpy(D).cuda()).cpu()

        def solve_fn(shells_aux, raw_full, nstates):
            return sh.solve_device(shells_aux, raw_full.cuda(), nstates)

        df, R, rng = sh.contract_coulomb_densities_4d_sharded(w.shells, w.shells_aux, w.densities,
                                                              raw_fn=raw_fn, solve_fn=solve_fn)
    finally:
        dist.destroy_process_group()
    assert rng == (0, len(w.shells_aux))
    R_ref = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    close(R, R_ref, 1e-13, atol=1e-12)
