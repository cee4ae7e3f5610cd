"""Autotuner of the three-center tile shapes.

The class kernels of the screened three-center contraction come in tile-shape
variants per class (L_ab, L_c) (see ``pa_tile_shape`` in pa_b200.h): the tile
of auxiliary shells, the bra units per step, the lanes that build one
triplet's integrals and the blocks per SM. This module times every class in
every variant on the current GPU -- class-timing mode, where the class
launches run one after another and each is timed with CUDA events -- and
writes the table that the library applies at start-up (``df3c_tiles.txt``
beside libpa_b200.so, or ``$PA_B200_TILE_TABLE``).

Selection (``choose``): for each class and variant, the ratio of its time to
variant 0's is averaged over the workloads (each workload weighs the same,
however long its step); a variant replaces variant 0 when that mean ratio is
below ``1 - margin`` and no single workload sees it above ``1 + margin``.
Variants whose shape equals a lower variant's run the same kernel and are
not candidates.

    python -m pysisyphus_addons.tune --workloads cfg2,cfg5 --out PATH

The workloads are the seeded synthetic molecules of
``pysisyphus_addons.common.synthetic`` (cfg2: 40 atoms, lmax 3 / lauxmax 4;
cfg5: 200 atoms, lmax 4 / lauxmax 5).
"""
from __future__ import annotations

import argparse
import json
import statistics
import time
from pathlib import Path

from . import _native as nat

DEFAULT_TABLE = Path(nat.LIB_PATH).resolve().parent / "df3c_tiles.txt"


def choose(times, margin=0.03, shapes=None):
    """times: {workload: {variant: {(lab, lc): ms}}} -> ({(lab, lc): variant},
    {(lab, lc): {variant: mean ratio to variant 0}}).

    A variant replaces variant 0 for a class when its time ratio to variant 0,
    averaged over the workloads, is below 1 - margin and no workload sees it
    above 1 + margin. shapes ({(lab, lc): {variant: shape}}, optional) drops
    variants whose shape equals a lower variant's: they run the same kernel,
    so their differences are timing noise. Classes missing from a workload's
    variant-0 run are decided by the other workloads."""
    ratios = {}
    for per_v in times.values():
        base = per_v.get(0, {})
        for v, cls in per_v.items():
            for key, ms in cls.items():
                if key in base and base[key] > 0:
                    ratios.setdefault(key, {}).setdefault(v, []).append(ms / base[key])
    table, mean = {}, {}
    for key, per_v in ratios.items():
        sh = (shapes or {}).get(key, {})
        distinct = [v for v in per_v if v == 0 or not any(
            sh.get(v) is not None and sh.get(v) == sh.get(u) for u in per_v if u < v)]
        mean[key] = {v: sum(per_v[v]) / len(per_v[v]) for v in distinct}
        ok = [v for v in distinct if v != 0 and mean[key][v] < 1.0 - margin and max(per_v[v]) < 1.0 + margin]
        table[key] = min(ok, key=lambda v: (mean[key][v], v)) if ok else 0
    return table, mean


def format_table(table, mean=None, header=()):
    lines = ["# three-center tile-shape variants per class (pysisyphus_addons.tune)"]
    lines += [f"# {h}" for h in header]
    lines.append("# L_ab L_c variant")
    for (lab, lc) in sorted(table):
        v = table[(lab, lc)]
        if v == 0:
            continue
        note = ""
        if mean and (lab, lc) in mean:
            note = "  # mean time ratio to variant 0: " + ", ".join(
                f"v{k} {r:.3f}" for k, r in sorted(mean[(lab, lc)].items()))
        lines.append(f"{lab} {lc} {v}{note}")
    return "\n".join(lines) + "\n"


def parse_table(text):
    """{(lab, lc): variant} of a table's text (the library's format)."""
    out = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].split()
        if not line:
            continue
        if len(line) != 3:
            raise ValueError(f"malformed tile-table line: {line}")
        lab, lc, v = (int(x) for x in line)
        out[(lab, lc)] = v
    return out


def class_times(orb, aux, dens, reps=3, variant=0):
    """{(lab, lc): median ms over reps} of one workload with every class in
    `variant` (device densities `dens`, a (nd, nbf, nbf) torch tensor)."""
    import torch

    nd, nbf = dens.shape[0], dens.shape[1]
    out = torch.empty(aux.nsph * nd, dtype=torch.float64, device=dens.device)
    lib = nat.load()
    stream = torch.cuda.current_stream().cuda_stream
    for lab in range(2 * nat.LMAX + 1):
        for lc in range(nat.LAUXMAX + 1):
            nat.set_tile_variant(lab, lc, variant)
    nat.set_class_timing(True)
    samples = {}
    try:
        # one untimed call: first launches of each kernel, allocations
        nat.check(lib.pa_df_2d(orb.handle, aux.handle, nd, nbf, dens.data_ptr(), nat.PA_LAYOUT_C,
                               out.data_ptr(), stream))
        for _ in range(reps):
            nat.check(lib.pa_df_2d(orb.handle, aux.handle, nd, nbf, dens.data_ptr(), nat.PA_LAYOUT_C,
                                   out.data_ptr(), stream))
            for lab, lc, ms in nat.get_class_times():
                samples.setdefault((lab, lc), []).append(ms)
    finally:
        nat.set_class_timing(False)
    return {k: statistics.median(v) for k, v in samples.items()}


def tune(workloads=("cfg2", "cfg5"), reps=3, margin=0.03, variants=None, log=print):
    """Times the workloads in every variant; returns (table, mean ratios, raw
    times). The current tile table is restored afterwards."""
    import numpy as np
    import torch

    from .common.synthetic import config_workload

    variants = list(range(nat.TILE_VARIANTS)) if variants is None else list(variants)
    saved = {(lab, lc): nat.get_tile_variant(lab, lc)
             for lab in range(2 * nat.LMAX + 1) for lc in range(nat.LAUXMAX + 1)}
    times = {}
    try:
        for key in workloads:
            t0 = time.time()
            w = config_workload(key)
            orb, aux = nat.Basis(w.shells, "orbital"), nat.Basis(w.shells_aux, "aux")
            dens = torch.from_numpy(np.ascontiguousarray(w.densities)).cuda()
            times[key] = {v: class_times(orb, aux, dens, reps, v) for v in variants}
            log(f"tune: {key} timed in {len(variants)} variants ({time.time() - t0:.1f} s)")
            del dens
            torch.cuda.empty_cache()
    finally:
        for (lab, lc), v in saved.items():
            nat.set_tile_variant(lab, lc, v)
    shapes = {(lab, lc): {v: tuple(sorted(nat.tile_shape(lab, lc, v).items())) for v in variants}
              for lab in range(2 * nat.LMAX + 1) for lc in range(nat.LAUXMAX + 1)}
    table, mean = choose(times, margin, shapes)
    return table, mean, times


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workloads", default="cfg2,cfg5")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--margin", type=float, default=0.03)
    ap.add_argument("--out", default=str(DEFAULT_TABLE))
    ap.add_argument("--report", default=None, help="JSON file for the raw class times")
    args = ap.parse_args(argv)
    import torch

    torch.cuda.set_device(0)
    workloads = [w for w in args.workloads.split(",") if w]
    if "cfg5" in workloads:
        # the 200-atom workload's settings (as its bench): exact Boys, metric shift
        nat.set_boys_mode("exact")
        nat.set_metric_shift(1e-7)
    table, mean, times = tune(workloads, args.reps, args.margin)
    props = torch.cuda.get_device_properties(0)
    header = [f"device: {props.name}, {props.multi_processor_count} SMs",
              f"workloads: {', '.join(workloads)}; {args.reps} timed calls per variant; margin {args.margin}"]
    Path(args.out).write_text(format_table(table, mean, header))
    print(f"tune: {sum(v != 0 for v in table.values())} of {len(table)} classes off variant 0 -> {args.out}")
    if args.report:
        rep = {"header": header,
               "table": {f"{a},{b}": v for (a, b), v in sorted(table.items())},
               "mean_ratio": {f"{a},{b}": {str(k): r for k, r in m.items()} for (a, b), m in sorted(mean.items())},
               "class_ms": {w: {str(v): {f"{a},{b}": ms for (a, b), ms in sorted(c.items())}
                                for v, c in per_v.items()} for w, per_v in times.items()}}
        Path(args.report).write_text(json.dumps(rep, indent=1))


if __name__ == "__main__":
    main()
