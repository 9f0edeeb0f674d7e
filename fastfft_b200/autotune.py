"""Per-shape schedule autotuner for the batched correlation.

The schedule of the batched reduced-size path has three knobs:
  * templates per launch (`SetTemplatesPerLaunch`): more templates per launch share each
    staged image column and fill the GPU with fewer, larger launches, but stage more
    template columns in shared memory and hold larger intermediates;
  * groups in flight (`SetPipelinedGroups`): with 2, consecutive groups alternate between two
    streams, so one group's row passes overlap the other's column pass and a group's
    intermediates (its row-pass and column-pass outputs) can stay in L2 instead of making a
    round trip through HBM;
  * templates per block of the fused column pass (`SetTemplatesPerBlock`): each block stages
    one image column and this many template columns; more per block share the staged column
    and cost shared memory and a longer last wave.
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
PER_BLOCK_CANDIDATES = (0, 2, 4, 6, 8, 12, 16)            # 0: the built-in choice per length


def _key(ft, n_templates, sizes):
    import torch

    fi, fo, io = ft.ReturnFwdInputDimensions(), ft.ReturnFwdOutputDimensions(), ft.ReturnInvOutputDimensions()
    shape = "" if sizes is None else "|" + ",".join(f"{x}x{y}" for x, y in sorted(set(map(tuple, sizes))))
    return f"{torch.cuda.get_device_name()}|{fi[:3]}|{fo[:3]}|{io[:3]}|{n_templates}{shape}"


def tune(ft, inputs, image, outputs, sizes=None, candidates=CANDIDATES, pipelined=PIPELINED_CANDIDATES,
         per_block=PER_BLOCK_CANDIDATES, reps=3, cache_path=None):
    """Pick the (templates per launch, groups in flight) schedule with the lowest time for this
    batch, then the templates per block for it; leaves the plan set to the result and returns
    the templates per launch.

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
            ft.SetTemplatesPerBlock(cache[key].get("templates_per_block", 0))
            return ft.TemplatesPerLaunch()

    def run():
        if sizes is None:
            ft.FwdImageInvFFTMany(inputs, image, outputs)
        else:
            ft.FwdImageInvFFTManySized(inputs, sizes, image, outputs)

    def measure():
        run()  # warm-up (also allocates the work buffer for this schedule)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    timings = {}
    ft.SetTemplatesPerBlock(0)
    schedule = [(1, g) for g in candidates] + [(2, g) for g in pipelined]
    for groups, g in schedule:
        ft.SetPipelinedGroups(groups)
        ft.SetTemplatesPerLaunch(g)
        eff = (ft.PipelinedGroups(), ft.TemplatesPerLaunch(), 0)
        if eff not in timings:
            timings[eff] = measure()
    best = min(timings, key=timings.get)
    ft.SetPipelinedGroups(best[0])
    ft.SetTemplatesPerLaunch(best[1])
    builtin = ft.TemplatesPerBlock()
    for b in per_block:
        if b == 0:
            continue
        ft.SetTemplatesPerBlock(b)
        eff = (best[0], ft.TemplatesPerLaunch(), ft.TemplatesPerBlock())
        if eff[1] != best[1] or eff[2] == builtin or eff in timings:
            continue          # (shared memory lowered the templates per launch, or the same choice)
        timings[eff] = measure()
    best = min(timings, key=timings.get)
    ft.SetPipelinedGroups(best[0])
    ft.SetTemplatesPerBlock(best[2])
    ft.SetTemplatesPerLaunch(best[1])
    tune.last_timings = {f"{k[0]}x{k[1]}" + (f"/{k[2]}" if k[2] else ""): v for k, v in timings.items()}
    if cache_path:
        cache[key] = {"groups": best[0], "templates_per_launch": best[1], "templates_per_block": best[2],
                      "ms": tune.last_timings}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, default=str)
    return best[1]


tune.last_timings = {}
