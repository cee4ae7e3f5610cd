"""One molecule's Coulomb tensor sharded over ranks by auxiliary shells.

The reference runs the three-center loop with one OpenMP thread per auxiliary
shell; every thread owns its rows df(k, :) (diabatization/intor.f90:117-126,
dynamic schedule). Across GPUs the same independence gives the partition:

  1. the auxiliary shells are split into consecutive ranges, one per rank,
     balanced by the modelled flops of their surviving triplets
     (pysisyphus_addons.flops, from the Schwarz vectors);
  2. each rank contracts all surviving (ab|c) of its range with the densities
     (the raw contraction, before the metric) -- its rows of df;
  3. one all-gather assembles the raw contraction on every rank (naux x ndens
     doubles: 3.9 MB at 13400 auxiliary functions and 36 densities);
  4. every rank then runs the metric chain and the solve itself (replicated:
     (P|Q) is at most a few GB, its factorization a fraction of the
     three-center time).

The gathered raw contraction is the same on every rank, so every rank returns
the same df and tensor. The collective is the only exchange; ranks use
torch.distributed (NCCL for device tensors, gloo for host tensors).
"""

import numpy as np

from pysisyphus_addons import _native as nat
from pysisyphus_addons import flops as fl
from pysisyphus_addons.common.shells import Shells


def aux_shell_costs(shells, shells_aux, q_bra, q_aux, nd, thresh=float(np.float32(1e-10))):
    """Modelled flops of the surviving triplets of every auxiliary shell
    (the per-unit model of pysisyphus_addons.flops)."""
    n = len(shells)
    La = np.array([s.L for s in shells])
    Pa = np.array([s.nprims for s in shells])
    ia, ib = np.tril_indices(n)  # packed a(a+1)/2 + b order of the bra Schwarz vector
    lab = La[ia] + La[ib]
    units = (Pa[ia] * Pa[ib]).astype(float)
    qb = np.asarray(q_bra)
    costs = np.zeros(len(shells_aux))
    labs = np.unique(lab)
    for k, (c, qc) in enumerate(zip(shells_aux, np.asarray(q_aux))):
        surv = qb * qc >= thresh
        tot = 0.0
        for l in labs:
            m = surv & (lab == l)
            if m.any():
                tot += fl.triple_flops(int(l), c.L, nd) * float(units[m].sum()) * c.nprims
        costs[k] = tot
    return costs


def partition_aux_shells(costs, nranks):
    """Consecutive ranges [lo, hi) of auxiliary shells, one per rank, whose
    summed costs are as even as a prefix split allows: rank r's range ends at
    the shell where the running cost crosses (r + 1) / nranks of the total
    (the nearer side of the crossing). Ranges may be empty when there are
    fewer shells than ranks; together they cover every shell once."""
    costs = np.asarray(costs, dtype=float)
    n = len(costs)
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, nranks):
        target = total * r / nranks
        j = int(np.searchsorted(cum, target))  # first prefix end with cum >= target
        if j > 0 and abs(cum[j - 1] - target) <= abs(cum[min(j, n)] - target):
            j -= 1
        cuts.append(min(max(j, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(nranks)]


def shard_rows(shells_aux, ranges):
    """Spherical row offsets of each range in the full auxiliary basis."""
    sizes = np.array([2 * s.L + 1 for s in shells_aux])
    off = np.concatenate([[0], np.cumsum(sizes)])
    return [(int(off[lo]), int(off[hi])) for lo, hi in ranges]


def gather_aux_rows(local, counts, group=None):
    """All-gather of row blocks: `local` is this rank's (ndens, n_local)
    tensor (the column-major naux_local x ndens block), counts[r] the rows of
    rank r. Returns the (ndens, sum(counts)) tensor -- the full column-major
    naux x ndens raw contraction -- on every rank."""
    import torch
    import torch.distributed as dist

    nd = local.shape[0]
    width = max(max(counts), 1)
    padded = torch.zeros((nd, width), dtype=local.dtype, device=local.device)
    padded[:, : local.shape[1]] = local
    parts = [torch.empty_like(padded) for _ in counts]
    dist.all_gather(parts, padded.contiguous(), group=group)
    return torch.cat([p[:, :c] for p, c in zip(parts, counts)], dim=1).contiguous()


def raw_contraction_device(shells, shells_aux_sub, dens_dev, stream=None):
    """The raw contraction sum (ab|c) Dsym of the auxiliary shells of a sub-basis
    on the current device: a (ndens, naux_sub) device tensor (column-major
    naux_sub x ndens)."""
    import torch

    nd, nbf = dens_dev.shape[0], dens_dev.shape[1]
    naux = shells_aux_sub.sph_size
    out = torch.zeros((nd, naux), dtype=torch.float64, device=dens_dev.device)
    if naux == 0 or nd == 0:
        return out
    stream = stream or torch.cuda.current_stream().cuda_stream
    orb = nat.Basis(shells, "orbital")
    aux = nat.Basis(shells_aux_sub, "aux")
    nat.set_skip_metric(1)
    try:
        nat.check(nat.load().pa_df_2d(orb.handle, aux.handle, nd, nbf, dens_dev.data_ptr(), nat.PA_LAYOUT_C,
                                      out.data_ptr(), stream))
    finally:
        nat.set_skip_metric(0)
    return out


def solve_device(shells_aux, raw_full, nstates, stream=None):
    """(df, Coulomb tensor) of a gathered raw contraction (device tensors) by
    pa_df_solve: metric, Cholesky factor, L^-1 raw, tensor."""
    import torch

    nd, naux = raw_full.shape
    stream = stream or torch.cuda.current_stream().cuda_stream
    aux = nat.Basis(shells_aux, "aux")
    df = torch.empty((nd, naux), dtype=torch.float64, device=raw_full.device)
    R = torch.empty(max(nstates, 1) ** 4, dtype=torch.float64, device=raw_full.device)
    nat.check(nat.load().pa_df_solve(aux.handle, nd, raw_full.data_ptr(), df.data_ptr(), nstates, R.data_ptr(),
                                     stream))
    return df, R


def contract_coulomb_densities_4d_sharded(shells, shells_aux, densities, group=None, raw_fn=None,
                                          solve_fn=None, costs=None):
    """Coulomb tensor of one molecule with its auxiliary shells sharded over
    the ranks of `group` (torch.distributed must be initialized). Returns
    (df[naux, ndens], R[ns, ns, ns, ns]) as numpy arrays on every rank, plus
    this rank's range of auxiliary shells.

    raw_fn(shells, shells_aux_sub, densities) -> (ndens, naux_sub) tensor and
    solve_fn(shells_aux, raw_full, nstates) -> (df, R) default to the device
    path (pa_df_2d with the metric skipped, and pa_df_solve); `costs` are the
    per-auxiliary-shell weights of the partition (default: the flops model on
    the device Schwarz vectors)."""
    import torch
    import torch.distributed as dist

    from pysisyphus_addons.intor import intor as sch

    D = np.ascontiguousarray(densities, dtype=np.float64)
    nd = D.shape[0]
    nstates = int(round((np.sqrt(8 * nd + 1) - 1) / 2))
    if nstates * (nstates + 1) // 2 != nd:
        raise ValueError("ndens must equal nstates (nstates + 1) / 2")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if costs is None:
        costs = aux_shell_costs(shells, shells_aux, sch.int_schwarz_bra(shells), sch.int_schwarz_aux(shells_aux), nd)
    ranges = partition_aux_shells(costs, world)
    rows = shard_rows(shells_aux, ranges)
    lo, hi = ranges[rank]
    sub = Shells(shells_aux.shells[lo:hi])
    if raw_fn is None:
        dens_dev = torch.from_numpy(D).cuda()
        raw_fn = lambda s, x, _d: raw_contraction_device(s, x, dens_dev)  # noqa: E731
    local = raw_fn(shells, sub, D)
    raw_full = gather_aux_rows(local, [b - a for a, b in rows], group)
    if solve_fn is None:
        solve_fn = solve_device
    df, R = solve_fn(shells_aux, raw_full, nstates)
    df = df.cpu().numpy() if hasattr(df, "cpu") else np.asarray(df)
    R = R.cpu().numpy() if hasattr(R, "cpu") else np.asarray(R)
    return (df.reshape(nd, -1).T.copy(order="F"), R.reshape((nstates,) * 4, order="F"), (lo, hi))
