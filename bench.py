"""Benchmark of the density-fitting Coulomb-tensor path on B200.

One step = one full Coulomb tensor of the 40-atom workload (lmax 3 / lauxmax 4,
8 states, 36 densities) on the device: Schwarz screening, class sorting,
density folding, metric + Cholesky, screened 3c2e contraction, L^-1 df and
the tensor assembly. Inputs (basis handles, densities) are resident in HBM
when the timed region starts; the densities (133 MB) exceed the 126 MB L2.

metric: surviving spherical 3c2e integrals per second (the integrals the
reference evaluates after Schwarz screening, diabatization/intor.f90:126-151).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

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

METRIC = "3c2e ints/s (Coulomb tensor, FP64 plain path)"
UNIT = "ints/s"
CONFIG_KEY = "cfg2"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=CONFIG_KEY)
    ap.add_argument("--boys", default="reference", choices=["reference", "exact"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="device steps only (for ncu): no e2e, CPU baseline, FP64 probe or clocks")
    return ap.parse_args()


def workload_config(key, w, nd):
    from pysisyphus_addons.common.synthetic import CONFIGS

    c = CONFIGS[key]
    return {
        "workload": f"df_coulomb_tensor_{c['natoms']}atoms_lmax{c['lmax']}_lauxmax{c['lauxmax']}_{c['nstates']}states",
        "natoms": c["natoms"],
        "lmax": c["lmax"],
        "lauxmax": c["lauxmax"],
        "nstates": c["nstates"],
        "ndens": nd,
        "nbf": w.shells.sph_size,
        "naux": w.shells_aux.sph_size,
        "nshells": len(w.shells),
        "nshells_aux": len(w.shells_aux),
        "screen_thresh": "float32(1e-10)",
        "l2": "inputs larger than L2 (densities %.0f MB > 126 MB)" % (w.densities.nbytes / 1e6),
    }


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


def cpu_baseline(w, nints, steps=1):
    import oracle

    oracle.set_boys_mode("reference")
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    dt = (time.perf_counter() - t0) / steps
    return {"value": nints / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} full Coulomb tensor(s) of the same workload, C++ OpenMP restatement of the "
                      f"reference driver (oracle/), {dt:.2f} s each"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from pysisyphus_addons.common.synthetic import config_workload

    import oracle

    w = config_workload(args.config, seed=0)
    nd = len(w.densities)
    oracle.set_boys_mode("reference")
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    for _ in range(args.warmup):
        oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    nints = oracle.last_stats()["nints"]
    value = nints / dt
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": workload_config(args.config, w, nd), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "every step one full Coulomb tensor of the workload; C++ OpenMP restatement of "
                                   "the reference driver (the Fortran reference and its generated integral "
                                   "kernels cannot be built here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    from pysisyphus_addons import _native as nat
    from pysisyphus_addons import flops as fl
    from pysisyphus_addons.common.synthetic import config_workload
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
    w = config_workload(args.config, seed=rank)
    nd = len(w.densities)
    ns = w.nstates
    nbf = w.shells.sph_size
    orb = nat.Basis(w.shells, "orbital")
    aux = nat.Basis(w.shells_aux, "aux")
    ntrip_all, ntrip, nints = nat.count_triplets(orb, aux)
    qb = sch.int_schwarz_bra(w.shells)
    qa = sch.int_schwarz_aux(w.shells_aux)
    flops_3c, ntrip_model, nints_model = fl.model(w.shells, w.shells_aux, qb, qa, nd)
    assert ntrip_model == ntrip and nints_model == nints, (ntrip_model, ntrip, nints_model, nints)

    dens = torch.from_numpy(np.ascontiguousarray(w.densities)).cuda()
    out = torch.empty(ns**4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    lib = nat.load()

    def step():
        nat.check(lib.pa_df_4d(orb.handle, aux.handle, nd, nbf, dens.data_ptr(), nat.PA_LAYOUT_C, ns,
                               out.data_ptr(), stream.cuda_stream))

    if args.profile:
        for _ in range(args.warmup + args.steps):
            step()
        torch.cuda.synchronize()
        return
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    ms3c, launches, launches3c, phases = [], 0, 0, []
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        step()
        st = nat.get_stats()
        ms3c.append(st["ms_3c"])
        phases.append({k: st[k] for k in ("ms_screen", "ms_bra", "ms_metric", "ms_3c", "ms_solve")})
        launches += st["kernel_launches"]
        launches3c += st["launches_3c"]
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    elapsed = t_start.elapsed_time(t_end) / 1e3
    if world > 1:
        t = torch.tensor([elapsed], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        n = torch.tensor([float(nints)], device="cuda", dtype=torch.float64)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        total_ints = float(n.item())
    else:
        total_ints = float(nints)
    step_s = elapsed / args.steps
    value = total_ints / step_s

    # end to end: the public Python API with pinned host densities (H2D + D2H inside)
    e2e = None
    if not args.no_e2e:
        pinned = torch.from_numpy(np.ascontiguousarray(w.densities)).pin_memory().numpy()
        for _ in range(2):
            R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, pinned)
        torch.cuda.synchronize()
        barrier()
        iters = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ti = time.perf_counter()
            R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, pinned)
            iters.append((time.perf_counter() - ti) * 1e3)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / args.steps
        if world > 1:
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        keep = [a for a in w.shells.as_arrays(fortran=True)] + [a for a in w.shells_aux.as_arrays(fortran=True)]
        h2d = int(pinned.nbytes + sum(a.nbytes for a in keep))
        e2e = {"value": total_ints / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": int(R.nbytes), "ms_per_step": e2e_s * 1e3,
               "ms_per_call": [round(x, 3) for x in iters]}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peak = fp64_peak_tflops(torch)
    ms3 = statistics.mean(ms3c)
    achieved = flops_3c / (ms3 / 1e3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": dict(workload_config(args.config, w, nd), boys_mode=args.boys,
                       parallelism=f"independent molecules x{world}" if world > 1 else "single GPU"),
        "roofline": {"bound": "fp64", "kernel": "k_df3c (all classes) + ordered reduction",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": "FP64 GEMM (torch.matmul float64 8192^3) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "flops_per_step_3c": flops_3c, "ms_3c": ms3, "traffic": None},
        "phases_ms": {k: statistics.mean(p[k] for p in phases) for k in phases[0]},
        "screening": {"triplets": ntrip_all, "computed": ntrip, "ints": nints},
        "gpu_launches": launches,
        "gpu_launches_3c": launches3c,
        "clocks": clk,
    }
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, nints)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
