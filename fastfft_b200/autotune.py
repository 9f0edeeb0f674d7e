"""Per-shape schedule autotuner for the batched correlation.

The schedule of the batched reduced-size path has two knobs:
  * templates per launch (`SetTemplatesPerLaunch`): more templates per launch share each
    staged image column and fill the GPU with fewer, larger launches, but stage more
    template columns in shared memory and hold larger intermediates;
  * groups in flight (`SetPipelinedGroups`): with 2, consecutive groups alternate between two
    streams, so one group's row passes overlap the other's column pass and a group's
    intermediates (its row-pass and column-pass outputs) can stay in L2 instead of making a
    round trip through HBM.
The best schedule depends on the correlation size, the template sizes and the GPU; `tune`
measures the candidates on the caller's own plan and batch with CUDA events and keeps the
fastest.  Results can be cached in a JSON file keyed by the device name, the plan's sizes and
the batch.
"""
from __future__ import annotations

import json
import os

CANDIDATES = (8, 16, 32, 64)                              # one group in flight
PIPELINED_CANDIDATES = (4, 6, 8, 12, 16, 24, 32)          # two groups in flight


def _key(ft, n_templates, sizes):
    import torch

    fi, fo, io = ft.ReturnFwdInputDimensions(), ft.ReturnFwdOutputDimensions(), ft.ReturnInvOutputDimensions()
    shape = "" if sizes is None else "|" + ",".join(f"{x}x{y}" for x, y in sorted(set(map(tuple, sizes))))
    return f"{torch.cuda.get_device_name()}|{fi[:3]}|{fo[:3]}|{io[:3]}|{n_templates}{shape}"


def tune(ft, inputs, image, outputs, sizes=None, candidates=CANDIDATES, pipelined=PIPELINED_CANDIDATES, reps=3,
         cache_path=None):
    """Pick the (templates per launch, groups in flight) schedule with the lowest time for this
    batch; leaves the plan set to it and returns the templates per launch.

    inputs / outputs: the batch as it will be run (the outputs are overwritten); image: one
    image spectrum; sizes: per-template (x, y) for uneven batches.  `pipelined` may be empty
    to tune templates per launch alone.
    """
    import torch

    key = _key(ft, len(inputs), sizes)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            ft.SetPipelinedGroups(cache[key]["groups"])
            ft.SetTemplatesPerLaunch(cache[key]["templates_per_launch"])
            return ft.TemplatesPerLaunch()

    def run():
        if sizes is None:
            ft.FwdImageInvFFTMany(inputs, image, outputs)
        else:
            ft.FwdImageInvFFTManySized(inputs, sizes, image, outputs)

    timings = {}
    schedule = [(1, g) for g in candidates] + [(2, g) for g in pipelined]
    for groups, g in schedule:
        ft.SetPipelinedGroups(groups)
        ft.SetTemplatesPerLaunch(g)
        eff = (ft.PipelinedGroups(), ft.TemplatesPerLaunch())
        if eff in timings:
            continue
        run()  # warm-up (also allocates the work buffer for this schedule)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        timings[eff] = e0.elapsed_time(e1) / reps
    best = min(timings, key=timings.get)
    ft.SetPipelinedGroups(best[0])
    ft.SetTemplatesPerLaunch(best[1])
    tune.last_timings = {f"{k[0]}x{k[1]}": v for k, v in timings.items()}
    if cache_path:
        cache[key] = {"groups": best[0], "templates_per_launch": best[1], "ms": tune.last_timings}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, default=str)
    return best[1]


tune.last_timings = {}
