"""Per-shape schedule autotuner for the batched correlation.

The schedule knob of the batched reduced-size path is the number of templates per launch
(`SetTemplatesPerLaunch`): more templates per launch share each staged image column and
fill the GPU with fewer, larger launches, but stage more template columns in shared
memory, which can cost occupancy.  The best value depends on the correlation size, the
template size and the GPU; `tune` measures the candidates on the caller's own plan with
CUDA events and keeps the fastest.  Results can be cached in a JSON file keyed by the
device name and the plan's sizes.
"""
from __future__ import annotations

import json
import os

CANDIDATES = (8, 16, 32, 64)


def _key(ft, n_templates):
    import torch

    fi, fo, io = ft.ReturnFwdInputDimensions(), ft.ReturnFwdOutputDimensions(), ft.ReturnInvOutputDimensions()
    return f"{torch.cuda.get_device_name()}|{fi[:3]}|{fo[:3]}|{io[:3]}|{n_templates}"


def tune(ft, inputs, image, outputs, sizes=None, candidates=CANDIDATES, reps=3, cache_path=None):
    """Pick the templates-per-launch value with the lowest time for this batch; returns it.

    inputs / outputs: the batch as it will be run (the outputs are overwritten); image: one
    image spectrum.  The plan is left set to the chosen value.
    """
    import torch

    key = _key(ft, len(inputs))
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            ft.SetTemplatesPerLaunch(cache[key]["templates_per_launch"])
            return ft.TemplatesPerLaunch()

    def run():
        if sizes is None:
            ft.FwdImageInvFFTMany(inputs, image, outputs)
        else:
            ft.FwdImageInvFFTManySized(inputs, sizes, image, outputs)

    timings = {}
    for g in candidates:
        ft.SetTemplatesPerLaunch(g)
        eff = ft.TemplatesPerLaunch()
        if eff in timings:
            continue
        run()  # warm-up (also allocates the work buffer for this value)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        timings[eff] = e0.elapsed_time(e1) / reps
    best = min(timings, key=timings.get)
    ft.SetTemplatesPerLaunch(best)
    if cache_path:
        cache[key] = {"templates_per_launch": best, "ms": timings}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, default=str)
    return best
