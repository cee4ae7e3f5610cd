"""Benchmark of the density-fitting Coulomb-tensor path on B200.

Default (the headline line): the 200-atom cluster (lmax 4 / lauxmax 5, 8
states, 36 densities, 4950 basis / 13400 auxiliary functions). One step = one
full Coulomb tensor on the device: Schwarz screening, class sorting, density
folding, metric + Cholesky, screened 3c2e contraction, L^-1 df and the tensor
assembly. Two forms run back to back on the same inputs:

  - the plain FP64 form (pa_df_4d, precision fp64);
  - the headline form, mixed precision + batched (pa_df_4d_batch over the
    molecule, recorded once as a CUDA graph; FP32 recurrences for triplets
    whose Schwarz bound is below 1e-6).

`value` is the headline form's throughput; `forms` gives both forms' times,
their ratio and the max-abs / relative error of the headline form's tensor
against the FP64 form's. Inputs (basis handles, densities) are resident in
HBM when the timed region starts; the densities (7 GB) exceed the 126 MB L2.

metric: surviving spherical 3c2e integrals per second (the integrals the
reference evaluates after Schwarz screening, diabatization/intor.f90:126-151).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                  [--config cfg5|cfg2|cfg1|cfg4] [--form headline|fp64|mixed]

--config cfg2 is the 40-atom workload (lmax 3 / lauxmax 4), cfg4 the batch of
64 molecules (5-60 atoms, 4-16 states) run through pa_df_4d_batch (one CUDA
graph per step; --sequential: one pa_df_4d call per molecule). cfg5 and cfg4
use the exact Boys function and a 1e-7 diagonal shift of the metric: with the
reference's Boys interpolation their auxiliary metrics are indefinite and the
Cholesky fails (the reference ignores that failure). --form fp64 / mixed
measure a single form through pa_df_4d.

--impl reference times the reference's CPU algorithm (the C++ OpenMP
restatement under oracle/, as the Fortran reference cannot be built here) on
the host cores with the same workload and metric.

Under torchrun (N > 1) every rank evaluates its own molecule (same generator,
seed = rank): independent objects, no data-path collective, weak scaling.
"""

import argparse
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "pysisyphus-addons_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

UNIT = "ints/s"
CONFIG_KEY = "cfg5"
# the metric as named by the headline measurement
HEADLINE_METRIC = "3c2e ints/s and Coulomb-tensor time at \u22641e-9 err: mixed+batched vs FP64 GPU"
FP32_THRESH = 1e-6
# workloads whose auxiliary metric needs the exact Boys function and a shift
SHIFTED = {"cfg5": 1e-7, "cfg4": 1e-7}
# DRAM bytes (read + write) of the three-center family (k_df3c classes and
# reductions) per step, from ncu (dram__bytes_read.sum + dram__bytes_write.sum,
# -k regex:k_df3c) on the 40-atom step: 630.3 MB read + 0.3 MB written. The
# 200-atom value is that capture scaled by the model flops of the two steps
# (3.992e12 / 3.613e10): the traffic is the folded densities G re-read per
# auxiliary tile, which grows with the surviving triplets as the flops do.
TRAFFIC_3C = {"cfg2": 630.6e6, "cfg5": 630.6e6 * 3.992e12 / 3.613e10}
TRAFFIC_NOTE = {"cfg2": "ncu capture of this step (40 launches)",
                "cfg5": "40-atom ncu capture scaled by model flops (no full-size multi-metric capture)"}


def single_molecule(args):
    return args.config in ("cfg1", "cfg2", "cfg5")


def headline(args):
    """The headline measurement: mixed + batched against the plain FP64 form."""
    return single_molecule(args) and args.form == "headline"


def metric_name(args):
    if headline(args):
        return HEADLINE_METRIC
    if args.config == "cfg4":
        form = "mixed precision" if args.precision == "mixed" else "FP64 plain"
        path = "Coulomb tensors of the batch, one call per molecule" if args.sequential else "batched Coulomb tensors"
    else:
        form = {"mixed": "mixed precision", "mixed_split": "mixed precision, split-BF16 tensor-core product"}.get(
            args.form, "FP64 plain")
        path = "Coulomb tensor"
    if args.screening == "qvl":
        form += ", QVL screening"
    return f"3c2e ints/s ({path}, {form} path)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 5 for the 200-atom workload and the batch, 10 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=CONFIG_KEY, choices=["cfg1", "cfg2", "cfg5", "cfg4"])
    ap.add_argument("--form", default="headline", choices=["headline", "fp64", "mixed", "mixed_split"],
                    help="single-molecule workloads: headline = FP64 plain and both mixed + batched forms back "
                         "to back (value = mixed + batched); fp64 / mixed / mixed_split = one form through "
                         "pa_df_4d (mixed_split: weak triplets on the split-BF16 tensor-core kernels)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="cfg4: precision of the batch")
    ap.add_argument("--boys", default=None, choices=["reference", "exact"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision-report", action="store_true",
                    help="per-tensor errors and times of the precision form against the FP64 path "
                         "(and against the committed oracle fixture for the 40-atom workload)")
    ap.add_argument("--screening", default="schwarz", choices=["schwarz", "qvl"],
                    help="triplet estimate: schwarz (the reference's) or qvl (qvl_estimate); with qvl the "
                         "integral count follows the QVL set and the Schwarz-based flops model (roofline) "
                         "is not reported")
    ap.add_argument("--sequential", action="store_true",
                    help="cfg4: one pa_df_4d call per molecule (the reference's way) instead of the batched form")
    ap.add_argument("--profile", action="store_true",
                    help="device steps only (for ncu): no e2e, CPU baseline, FP64 probe or clocks")
    ap.add_argument("--std", action="store_true",
                    help="the sTDDFT tensors instead (int_df1c, int_eri2c, int_df2c_mo over 20 occupied + 40 "
                         "virtual orbitals) on the chosen workload; one step = the three tensors")
    ap.add_argument("--grid", action="store_true",
                    help="grid densities instead (f_eval_densities, one density on a cube grid of 64^3 points "
                         "around the molecule, blk_size 100, thresh 1e-8); one step = one evaluation")
    a = ap.parse_args()
    if a.boys is None:
        a.boys = "exact" if a.config in SHIFTED else "reference"
    if a.steps is None:
        a.steps = 5 if a.config in ("cfg5", "cfg4") else 10
    if not a.profile:
        a.warmup = max(3, a.warmup)  # at least three untimed warm-up steps
    return a


def workloads(args, rank=0):
    from pysisyphus_addons.common.synthetic import batch_workloads, config_workload

    if args.config == "cfg4":
        return batch_workloads(nmol=64)
    return [config_workload(args.config, seed=rank)]


def tile_report():
    """Which tile-shape variants the three-center classes ran in (the table
    the library applied at start-up, pysisyphus_addons.tune)."""
    from pysisyphus_addons import _native as nat

    off = {f"{a},{b}": v for a in range(2 * nat.LMAX + 1) for b in range(nat.LAUXMAX + 1)
           if (v := nat.get_tile_variant(a, b)) != 0}
    src = os.environ.get("PA_B200_TILE_TABLE")
    if src is None:
        table = Path(nat.LIB_PATH).resolve().parent / "df3c_tiles.txt"
        src = str(table.relative_to(ROOT)) if table.exists() and table.is_relative_to(ROOT) else (
            str(table) if table.exists() else "none (default shapes)")
    return {"table": src or "none (default shapes)", "classes_off_default": off}


def workload_config(args, ws):
    """The `config` object; both arms (ours and --impl reference) print the same one."""
    from pysisyphus_addons.common.synthetic import CONFIGS

    shift = SHIFTED.get(args.config, 0.0)
    base = {"boys_mode": args.boys, "screen_thresh": "float32(1e-10)", "screening": args.screening,
            "metric_shift": shift}
    if headline(args):
        base["forms"] = (f"fp64 plain (pa_df_4d) and mixed precision (FP32 recurrences below Schwarz bound "
                         f"{FP32_THRESH:g}) + batched (pa_df_4d_batch, CUDA graph); value = mixed + batched")
    elif args.config == "cfg4":
        base["precision"] = args.precision
    else:
        base["precision"] = args.form
    if shift:
        base["metric_shift_reason"] = ("auxiliary metric numerically singular for this workload "
                                       "(smallest eigenvalues ~ -1e-13 with exact Boys)")
    dens_mb = sum(w.densities.nbytes for w in ws) / 1e6
    base["l2"] = (f"inputs larger than L2 (densities {dens_mb:.0f} MB > 126 MB)" if dens_mb > 126 else
                  f"inputs smaller than L2 (densities {dens_mb:.1f} MB): not flushed between steps")
    if args.config == "cfg4":
        base["form"] = "one call per molecule" if args.sequential else "batched (pa_df_4d_batch, CUDA graph)"
        return dict(base, workload="df_coulomb_tensor_batch_64molecules_5to60atoms_lmax3_lauxmax4_4to16states",
                    nmol=len(ws), natoms_total=int(sum(len(w.mol.atomic_nums) for w in ws)),
                    nbf_total=int(sum(w.shells.sph_size for w in ws)),
                    naux_total=int(sum(w.shells_aux.sph_size for w in ws)),
                    ndens_total=int(sum(len(w.densities) for w in ws)))
    w = ws[0]
    c = CONFIGS[args.config]
    return dict(base,
                workload=f"df_coulomb_tensor_{c['natoms']}atoms_lmax{c['lmax']}_lauxmax{c['lauxmax']}_{c['nstates']}states",
                natoms=c["natoms"], lmax=c["lmax"], lauxmax=c["lauxmax"], nstates=c["nstates"],
                ndens=len(w.densities), nbf=w.shells.sph_size, naux=w.shells_aux.sph_size,
                nshells=len(w.shells), nshells_aux=len(w.shells_aux))



class Clocks:
    """SM clock and clock-event reasons sampled every 20 ms by a thread while
    the timed region runs (NVML reads only; nvidia-smi reports the same
    counters). Nothing here changes a GPU setting."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index):
        self.index = index
        self.nvml = None
        self.thread = None
        self.samples = []
        self.reasons = set()
        self.sm_max = None
        self.error = None

    def start(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.sm_max = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception as exc:  # no NVML: report that instead of clocks
            self.error = f"NVML unavailable: {exc}"
            return
        self.stop_flag = threading.Event()

        def loop():
            nv = self.nvml
            while not self.stop_flag.is_set():
                try:
                    self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    active = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for name, attr in self.REASONS:
                        if active & getattr(nv, attr):
                            self.reasons.add(name)
                except Exception as exc:
                    self.error = str(exc)
                    return
                self.stop_flag.wait(0.02)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not sampled"], "samples": 0}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        try:
            self.nvml.nvmlShutdown()
        except Exception:
            pass
        out = {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.sm_max,
               "reasons": sorted(self.reasons), "samples": len(self.samples)}
        if self.error:
            out["error"] = self.error
        return out


def fp64_peak_tflops(torch):
    """Measured FP64 GEMM throughput (torch.matmul float64, 8192^3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2 * n**3 / best / 1e12


def aggregate_over_ranks(dist, torch, elapsed_s, nints, device):
    """Whole-job figures of a multi-rank run: the slowest rank's time and the
    integrals of all ranks (every rank evaluates its own molecule)."""
    t = torch.tensor([float(elapsed_s)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(nints)], dtype=torch.float64, device=device)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


def oracle_sample(args, ws, budget_s=20.0):
    """Time the oracle (C++ OpenMP restatement of the reference driver) on a
    bounded sample of the workload. 8- and 40-atom workloads: one whole tensor.
    The batch: whole tensors of its first molecules while they fit the budget.
    200 atoms: every 200th auxiliary shell (17 shells of every angular momentum,
    on atoms across the cluster) against the full orbital basis -- all their
    surviving (ab|c), the metric and the solve; the bra Schwarz vector (an
    O(npairs) pass done once per tensor, ~0.1 % of a full CPU tensor) is
    computed on the first call and reused. Returns (ints/s, cores,
    description)."""
    import oracle

    from pysisyphus_addons.common.shells import Shells

    oracle.set_boys_mode(args.boys)
    oracle.set_metric_shift(SHIFTED.get(args.config, 0.0))
    oracle.set_screening(args.screening)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    if args.config in ("cfg1", "cfg2"):
        t0 = time.perf_counter()
        oracle.contract_coulomb_densities_4d(ws[0].shells, ws[0].shells_aux, ws[0].densities)
        dt = time.perf_counter() - t0
        n = oracle.last_stats()["nints"]
        return n / dt, threads, f"one full Coulomb tensor of the workload ({dt:.2f} s)"
    if args.config == "cfg4":
        done, ints, t_tot = 0, 0, 0.0
        for w in ws:
            t0 = time.perf_counter()
            oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
            t_tot += time.perf_counter() - t0
            ints += oracle.last_stats()["nints"]
            done += 1
            if t_tot > budget_s:
                break
        return ints / t_tot, threads, f"the first {done} molecules of the batch, whole tensors ({t_tot:.1f} s)"
    w = ws[0]
    sub = Shells(w.shells_aux.shells[::200])
    oracle.set_reuse_screening(1)
    try:
        oracle.contract_coulomb_densities_2d(w.shells, sub, w.densities)
        st = oracle.last_stats()
    finally:
        oracle.set_reuse_screening(0)
    dt = st["t_total"]
    return st["nints"] / dt, threads, (
        f"every 200th auxiliary shell ({len(sub)} of {len(w.shells_aux)}) against the full orbital basis: "
        f"all their surviving (ab|c), metric and solve ({dt:.1f} s; bra Schwarz vector reused)")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ws = workloads(args)
    steps = []
    for i in range(args.warmup + args.steps):
        v, threads, sample = oracle_sample(args, ws)
        if i >= args.warmup:
            steps.append(v)
    value = statistics.mean(steps) if steps else v
    line = {
        "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": workload_config(args, ws), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "every step: " + sample + "; C++ OpenMP restatement of the reference driver "
                                   "(the Fortran reference and its generated integral kernels cannot be built here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)



def aux_bench(args):
    """The adjacent paths: the sTDDFT tensors (--std) or grid densities (--grid)
    on the workload's molecule, timed with CUDA events over whole calls of the
    public functions (host arrays in and out: these paths have no device-buffer
    entry points). One JSON line; the time per step is the metric."""
    import torch

    from pysisyphus_addons import _native as nat
    from pysisyphus_addons.grid import grid
    from pysisyphus_addons.std import intor as std

    torch.cuda.set_device(0)
    nat.set_boys_mode(args.boys)
    nat.set_metric_shift(SHIFTED.get(args.config, 0.0))
    w = workloads(args)[0]
    if args.std:
        C = np.asfortranarray(w.mo_coeffs[:, :60])  # 20 occupied + 40 virtual orbitals

        def step():
            std.int_df1c(w.shells, w.shells_aux)
            std.int_eri2c(w.shells, w.shells_aux)
            std.int_df2c_mo(w.shells, w.shells_aux, C)
        metric, unit = "sTDDFT tensors (int_df1c + int_eri2c + int_df2c_mo, 20 occ + 40 virt MOs) per second", "sets/s"
        cfg = {"workload": workload_config(args, [w])["workload"], "nmos": 60, "boys_mode": args.boys}
    else:
        rng = np.random.default_rng(0)
        ncart = sum((s.L + 1) * (s.L + 2) // 2 for s in w.shells)
        Cc = rng.normal(size=(ncart, 20)) / np.sqrt(ncart)
        D = Cc @ Cc.T  # a symmetric positive semidefinite Cartesian density
        C = np.array([s.center for s in w.shells])
        lo, hi = C.min(0) - 3.0, C.max(0) + 3.0
        axes = [np.linspace(lo[d], hi[d], 64) for d in range(3)]
        X, Y, Z = np.meshgrid(*axes, indexing="ij")
        pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

        def step():
            grid.eval_density(w.shells, pts, D)
        metric, unit = "grid density points per second (f_eval_densities)", "points/s"
        cfg = {"workload": workload_config(args, [w])["workload"] + "_grid64cube", "npoints": len(pts),
               "ncart": ncart, "blk_size": 100, "thresh": 1e-8}
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if args.profile:
        for _ in range(args.steps):
            step()
        torch.cuda.synchronize()
        return
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    units = 1.0 if args.std else float(cfg["npoints"])
    line = {"metric": metric, "value": units / dt, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)", "config": cfg,
            "timing": "host wall clock around whole calls of the public host-array functions"}
    print(json.dumps(line), flush=True)


def precision_report(args):
    """Raw contraction, df = L^-1 raw and the Coulomb tensor of the FP64 path
    and of the precision form at several FP32 thresholds; max |difference| and
    its ratio to the tensor's largest element, plus median device times."""
    import torch

    from pysisyphus_addons import _native as nat

    torch.cuda.set_device(0)
    nat.set_boys_mode(args.boys)
    nat.set_metric_shift(SHIFTED.get(args.config, 0.0))
    w = workloads(args)[0]
    orb, aux = nat.Basis(w.shells, "orbital"), nat.Basis(w.shells_aux, "aux")
    nd, ns, nbf, naux = len(w.densities), w.nstates, w.shells.sph_size, w.shells_aux.sph_size
    dens = torch.from_numpy(np.ascontiguousarray(w.densities)).cuda()
    lib, s = nat.load(), torch.cuda.current_stream()

    def run(skip, tensor):
        nat.set_skip_metric(skip)
        try:
            if tensor:
                out = torch.empty(ns**4, dtype=torch.float64, device="cuda")
                nat.check(lib.pa_df_4d(orb.handle, aux.handle, nd, nbf, dens.data_ptr(), nat.PA_LAYOUT_C, ns,
                                       out.data_ptr(), s.cuda_stream))
            else:
                out = torch.empty(naux * nd, dtype=torch.float64, device="cuda")
                nat.check(lib.pa_df_2d(orb.handle, aux.handle, nd, nbf, dens.data_ptr(), nat.PA_LAYOUT_C,
                                       out.data_ptr(), s.cuda_stream))
            return out.cpu().numpy(), nat.get_stats()
        finally:
            nat.set_skip_metric(0)

    res = {}
    # mixed = FP32 recurrences inside the FP64 kernels; mixed_split = the weak
    # triplets on their own kernels with the split-BF16 tensor-core product
    for prec, thr, kernels in (("fp64", 0.0, 0), ("mixed", 1e-8, 0), ("mixed", 1e-6, 0), ("mixed", 1e-4, 0),
                               ("mixed_split", 1e-8, 1), ("mixed_split", 1e-6, 1), ("mixed_split", 1e-4, 1)):
        nat.set_precision("fp64" if prec == "fp64" else "mixed", thr)
        nat.set_mixed_kernels(kernels)
        t = {"raw": run(1, False)[0], "df": run(0, False)[0], "R": run(0, True)[0]}
        times = [run(0, True)[1] for _ in range(6)][2:]
        t["ms_total"] = statistics.median(x["ms_total"] for x in times)
        t["ms_3c"] = statistics.median(x["ms_3c"] for x in times)
        res[f"{prec}@{thr:g}"] = t
    nat.set_precision("fp64", 0.0)
    nat.set_mixed_kernels(0)
    base = res["fp64@0"]
    fixture = None
    if args.config == "cfg2" and args.boys == "reference":
        fixture = np.load(ROOT / "tests" / "golden" / "oracle_cfg2_reference.npz")

    def err(x, ref):
        d = float(np.abs(x - ref).max())
        return {"max_abs": d, "rel_of_max": d / float(np.abs(ref).max())}

    out = {}
    for k, t in res.items():
        row = {"ms_total": t["ms_total"], "ms_3c": t["ms_3c"],
               "vs_fp64_gpu": {n: err(t[n], base[n]) for n in ("raw", "df", "R")}}
        if fixture is not None:
            row["vs_fp64_oracle"] = {"raw": err(t["raw"].reshape(fixture["raw"].shape, order="F"), fixture["raw"]),
                                     "R": err(t["R"].reshape(fixture["R"].shape, order="F"), fixture["R"])}
        out[k] = row
    print(json.dumps({"workload": workload_config(args, [w]), "results": out}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.precision_report:
        precision_report(args)
        return
    if args.std or args.grid:
        aux_bench(args)
        return
    import torch
    import torch.distributed as dist

    from pysisyphus_addons import _native as nat
    from pysisyphus_addons import flops as fl
    from pysisyphus_addons.diabatization import intor as dia
    from pysisyphus_addons.intor import intor as sch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    nat.set_boys_mode(args.boys)
    nat.set_metric_shift(SHIFTED.get(args.config, 0.0))
    nat.set_screening(args.screening)
    ws = workloads(args, rank)
    orbs = [nat.Basis(w.shells, "orbital") for w in ws]
    auxs = [nat.Basis(w.shells_aux, "aux") for w in ws]
    nints, ntrip_all, ntrip, flops_3c = 0, 0, 0, 0.0
    for w, o, a in zip(ws, orbs, auxs):
        t_all, t_c, n_i = nat.count_triplets(o, a)
        nints += n_i
        ntrip_all += t_all
        ntrip += t_c
        if len(ws) == 1 and args.screening == "schwarz":
            qb = sch.int_schwarz_bra(w.shells)
            qa = sch.int_schwarz_aux(w.shells_aux)
            f, tm, im = fl.model(w.shells, w.shells_aux, qb, qa, len(w.densities))
            assert tm == t_c and im == n_i, (tm, t_c, im, n_i)
            flops_3c += f

    # densities live in pinned host memory (one copy per molecule) and on the device
    for w in ws:
        w.densities = torch.from_numpy(np.ascontiguousarray(w.densities)).pin_memory().numpy()
    dens = [torch.from_numpy(w.densities).cuda() for w in ws]
    ns = [w.nstates for w in ws]
    stream = torch.cuda.current_stream()
    lib = nat.load()
    step_stats = []  # statistics of every call of the last step

    def set_form(form):
        # mixed_split_batched: the weak triplets on their own kernels with the
        # split-BF16 tensor-core product (pa_set_mixed_kernels(1))
        nat.set_mixed_kernels(1 if form in ("mixed_split_batched", "mixed_split") else 0)
        if form in ("mixed", "mixed_split", "mixed_batched", "mixed_split_batched") or (
                form == "batched" and args.precision == "mixed"):
            nat.set_precision("mixed", FP32_THRESH)
        else:
            nat.set_precision("fp64")

    def make_step(kind, outs):
        """kind: "plain" (one pa_df_4d per molecule) or "batched" (pa_df_4d_batch)."""
        def step():
            step_stats.clear()
            if kind == "batched":
                nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True, stream=stream.cuda_stream)
                step_stats.append(nat.get_stats())
                return
            for o, a, d, k, out in zip(orbs, auxs, dens, ns, outs):
                nat.check(lib.pa_df_4d(o.handle, a.handle, d.shape[0], d.shape[1], d.data_ptr(),
                                       nat.PA_LAYOUT_C, k, out.data_ptr(), stream.cuda_stream))
                step_stats.append(nat.get_stats())
        return step

    # the measured forms, in order; the last one gives `value`
    if headline(args):
        forms = [("fp64", "plain"), ("mixed_split_batched", "batched"), ("mixed_batched", "batched")]
    elif args.config == "cfg4":
        forms = [("mixed" if args.precision == "mixed" else "fp64", "plain" if args.sequential else "batched")]
    else:
        forms = [(args.form, "plain")]
    outs = {name: [torch.empty(k**4, dtype=torch.float64, device="cuda") for k in ns] for name, _ in forms}

    if args.profile:
        for name, kind in forms:
            set_form(name)
            step = make_step(kind, outs[name])
            for _ in range(args.warmup + args.steps):
                step()
        torch.cuda.synchronize()
        nat.set_precision("fp64")
        nat.set_mixed_kernels(0)
        return

    clocks = Clocks(local)
    results = {}
    launches = 0
    total_ints = float(nints)
    for name, kind in forms:
        set_form(name)
        step = make_step(kind, outs[name])
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ms3c, phases, lc, lc3 = [], [], 0, 0
        barrier()
        torch.cuda.synchronize()
        if clocks.thread is None and clocks.error is None:
            clocks.start()
        t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for _ in range(args.steps):
            step()
            # the class kernels start while the density folding of later L_ab
            # classes still runs, so the span timed for them is folding + 3c
            ms3c.append(sum(st["ms_bra"] + st["ms_3c"] for st in step_stats))
            phases.append({k: sum(st[k] for st in step_stats)
                           for k in ("ms_screen", "ms_bra", "ms_metric", "ms_3c", "ms_solve")})
            lc += sum(st["kernel_launches"] for st in step_stats)
            lc3 += sum(st["launches_3c"] for st in step_stats)
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier()
        elapsed = t_start.elapsed_time(t_end) / 1e3
        if world > 1:
            elapsed, total_ints = aggregate_over_ranks(dist, torch, elapsed, nints, "cuda")
        launches += lc
        results[name] = {"kind": kind, "step_s": elapsed / args.steps, "value": total_ints / (elapsed / args.steps),
                         "ms3c": ms3c, "phases": phases, "launches": lc, "launches_3c": lc3}
    clk = clocks.stop()
    nat.set_precision("fp64")
    nat.set_mixed_kernels(0)
    head = results[forms[-1][0]]
    step_s, value = head["step_s"], head["value"]

    # errors of the headline form's tensor against the FP64 form's
    form_report = None
    if headline(args):
        Rf = outs["fp64"][0].cpu().numpy()
        Rm = outs["mixed_batched"][0].cpu().numpy()
        Rs = outs["mixed_split_batched"][0].cpu().numpy()
        dmax = float(np.abs(Rm - Rf).max())
        smax = float(np.abs(Rs - Rf).max())
        form_report = {
            "fp64_plain": {"ms_per_step": results["fp64"]["step_s"] * 1e3, "value": results["fp64"]["value"]},
            "mixed_batched": {"ms_per_step": step_s * 1e3, "value": value},
            "speedup_mixed_batched_vs_fp64": results["fp64"]["step_s"] / step_s,
            "tensor_err_vs_fp64": {"max_abs": dmax, "rel_of_max": dmax / float(np.abs(Rf).max())},
            "mixed_split_batched": {
                "kernels": "weak triplets on k_df3c_w: FP32 X build, split-BF16 tcgen05 product (3 slices per "
                           "operand, 6 products, FP32 accumulation per step, FP64 across steps)",
                "ms_per_step": results["mixed_split_batched"]["step_s"] * 1e3,
                "value": results["mixed_split_batched"]["value"],
                "speedup_vs_fp64": results["fp64"]["step_s"] / results["mixed_split_batched"]["step_s"],
                "tensor_err_vs_fp64": {"max_abs": smax, "rel_of_max": smax / float(np.abs(Rf).max())},
            },
            "fp32_thresh": FP32_THRESH,
        }

    # end to end through the reference-facing Python API: pinned host densities
    # copied in and the tensors copied out in every call
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(w.densities) for w in ws]  # already pinned
        e2e_form = forms[-1][0]
        set_form(e2e_form)
        batched_e2e = args.config == "cfg4" and not args.sequential
        if batched_e2e:
            host_out = [torch.empty(k**4, dtype=torch.float64).pin_memory() for k in ns]

            def call():
                for dd, hp in zip(dens, pinned):
                    dd.copy_(hp, non_blocking=True)
                nat.df_4d_batch(orbs, auxs, dens, ns, outs[e2e_form], use_graph=True, stream=stream.cuda_stream)
                for ho, o in zip(host_out, outs[e2e_form]):
                    ho.copy_(o, non_blocking=True)
                torch.cuda.synchronize()
                return host_out[0].numpy()
            api = "pysisyphus_addons._native.df_4d_batch (device buffers filled from pinned host memory)"
        else:
            arrs = [p.numpy() for p in pinned]

            def call():
                R = None
                for w, arr in zip(ws, arrs):
                    R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, arr)
                return R
            api = ("pysisyphus_addons.diabatization.intor.contract_coulomb_densities_4d (the reference's "
                   "function, host arrays; precision " + ("fp64" if e2e_form == "fp64" else "mixed") + "; the "
                   "basis arrays are compared on the host with the cached device copy of the basis, which the "
                   "first call built: no basis upload after it)")
        for _ in range(args.warmup):  # as many warm-up calls as the device loop
            call()
        torch.cuda.synchronize()
        barrier()
        iters = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ti = time.perf_counter()
            call()
            iters.append((time.perf_counter() - ti) * 1e3)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / args.steps
        nat.set_precision("fp64")
        if world > 1:
            e2e_s, _ = aggregate_over_ranks(dist, torch, e2e_s, 0, "cuda")
        h2d = int(sum(p.numpy().nbytes for p in pinned))
        d2h = int(sum(k**4 * 8 for k in ns))
        e2e = {"value": total_ints / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_s * 1e3, "api": api, "ms_per_call": [round(x, 3) for x in iters]}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    line = {
        "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": workload_config(args, ws),
        "screening": {"triplets": ntrip_all, "computed": ntrip, "ints": nints},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world > 1:
        line["ranks"] = f"independent molecules x{world} (seed = rank)"
    line["tiles"] = tile_report()
    if form_report:
        line["forms"] = form_report
    # roofline of the three-center family, timed in the plain form (its phase
    # events bracket the density folding + three-center span)
    plain = [n for n, k in forms if k == "plain" and len(ws) == 1]
    if plain and args.screening == "schwarz":
        r = results[plain[0]]
        peak = fp64_peak_tflops(torch)
        ms3 = statistics.mean(r["ms3c"])
        achieved = flops_3c / (ms3 / 1e3) / 1e12
        line["roofline"] = {
            "bound": "tensor", "pipe": "FP64 (DMMA m8n8k4 tensor cores + FP64 FMA)",
            "kernel": f"k_df3c<LAB,LC> (all classes) + ordered reduction in the {plain[0]} form, timed over the "
                      "folding + three-center span (k_bra_prep overlaps the first class launches)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "of measured: FP64 GEMM (torch.matmul float64 8192^3) in this run; "
                           "MEASURED_PEAKS.json has no FP64 figure",
            "flops_per_step_3c": flops_3c, "ms_bra_plus_3c": ms3,
            "traffic": TRAFFIC_3C.get(args.config), "traffic_unit": "bytes per step (family)",
            "traffic_source": TRAFFIC_NOTE.get(args.config)}
        line["phases_ms"] = {k: statistics.mean(p[k] for p in r["phases"]) for k in r["phases"][0]}
        line["gpu_launches_3c"] = r["launches_3c"]
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        v, threads, sample = oracle_sample(args, ws)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": sample + "; C++ OpenMP restatement of the reference driver (oracle/)"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
