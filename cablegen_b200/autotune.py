"""Autotuner of the engine's runtime parameters.

The knobs (cgb_set_option):

* ``sort_variant``  -- the digit pass of the radix sort: 0 ranks a 4096-key tile with warp
  match, 1 with eight ballots per digit (keys re-read from L2 for the local scatter), 2 keeps
  persistent CTAs that bulk-copy the next tile into shared memory while ranking the current one,
  3 is the ballot pass specialised for byte digits (full tiles without bounds tests, digits read
  from the one 32-bit word that holds them), 4 the same with 8192-key tiles of 512 threads (the
  tile-size knob), 5 is 4 ranking each key with one warp match in place of eight ballots;
* ``solve_variant`` -- 0 one thread per board, 1 the (board, empty cell) pairs of 32 boards
  spread over a warp;
* ``hash_load_pct`` -- load factor of the open-addressing index of solved layers (0 picks it by
  table size; a higher load means more probes, a lower one more memory and a lower L2 hit
  rate);
* ``move_window`` -- blocks of 1024 consecutive input boards whose moves share one repeat set
  in the move expansion (more blocks keep fewer repeats out of the sort, at the price of longer
  probes in a fuller set).

The digit width stays at 8 bits: the look-back words and the per-tile histograms grow with the
radix (2048 bins at 11 bits), which costs more than the pass it saves on 48 varying key bits.

`tune()` runs a short prefix of a workload once per candidate value, one knob at a time
(coordinate descent from the defaults), keeps the fastest device time, and caches the result
per GPU model and workload in a JSON file.
"""
from __future__ import annotations

import dataclasses
import json
import os
from typing import Dict, Optional

from . import configs, device

KNOBS = {
    "sort_variant": [4, 5, 3, 1, 0, 2],
    "solve_variant": [1, 0],
    "hash_load_pct": [0, 25, 45],
    "move_window": [1, 2, 4],
}

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "cablegen_b200", "autotune.json")


def _gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def _runner(workload: str, end_cap: int, precision: int):
    """A function that runs the workload prefix once and returns its device milliseconds."""
    w = configs.get(workload)
    forms = [dataclasses.replace(f, end_gen=min(f.end_gen, end_cap)) for f in w.formations]

    def run() -> float:
        device.set_rules(w.settings)
        if len(forms) > 1:
            _, _, st = device.batch(forms, precision=precision)
        else:
            f = forms[0]
            _, _, st = device.tablebase(f.initial, f.start, f.end_gen, f.start, f.winstates, precision)
        return float(st["total_ms"])
    return run


def tune(workload: str = "batch64", end_cap: int = 300, precision: int = 32, repeats: int = 2,
         cache: Optional[str] = DEFAULT_CACHE, force: bool = False) -> Dict:
    """Picks and applies the fastest value of every knob; returns {"params", "ms", "trials", "cached"}."""
    key = f"{_gpu_name()}|{workload}|{end_cap}|{precision}"
    if cache and not force and os.path.exists(cache):
        try:
            with open(cache) as f:
                entry = json.load(f).get(key)
        except (OSError, ValueError):
            entry = None
        if entry:
            for k, v in entry["params"].items():
                device.set_option(k, v)
            return dict(entry, cached=True)
    run = _runner(workload, end_cap, precision)
    run()  # warm-up: allocations, pools, first launches
    params = {k: device.get_option(k) for k in KNOBS}
    trials = []

    def measure() -> float:
        return min(run() for _ in range(repeats))

    best_ms = measure()
    trials.append({"params": dict(params), "ms": best_ms})
    for knob, values in KNOBS.items():
        start = params[knob]  # measured already, with the other knobs as they are now
        for v in values:
            if v == start:
                continue
            device.set_option(knob, v)
            ms = measure()
            trials.append({"params": dict(params, **{knob: v}), "ms": ms})
            if ms < best_ms:
                best_ms = ms
                params[knob] = v
            device.set_option(knob, params[knob])
    entry = {"params": params, "ms": best_ms, "trials": trials}
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            data = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    data = json.load(f)
            data[key] = entry
            with open(cache, "w") as f:
                json.dump(data, f, indent=1)
        except (OSError, ValueError):
            pass
    return dict(entry, cached=False)
