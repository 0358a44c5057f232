"""Autotuner of the Sigma kernels' launch shapes (no counterpart in the reference, whose evaluator is a CPU loop).

The panel kernel's work units (runs of ``batch x unit_batches`` pole tuples of one path class) trade load
balance against per-unit set-up; the wide-chain kernel's units and its CTAs per SM trade the same against
occupancy.  ``tune_sigma`` times the Sigma evaluation of a set of topologies on a device-resident G for each
candidate value, one parameter at a time (coordinate descent from the current setting), keeps the fastest,
and records the choice in a JSON cache keyed by the device, the DLR rank, the pole count, the block
structure and the topologies, so later runs of the same configuration start from it (``apply_cached``).
Results do not depend on the choice in the ordered summation mode; in the fast mode only the order of the
atomic additions changes.
"""

import json
import os

import numpy as np

CANDIDATES = {
    "unit_batches": (1, 2, 4, 8, 16),
    "wide_unit_tuples": (1, 4, 16),
    "wide_ctas_per_sm": (1, 2),
}


def default_cache_path():
    return os.environ.get("XCA_TUNING_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "xca_b200", "tuning.json"))


def config_key(evaluator, terms, device_name=None):
    if device_name is None:
        try:
            import torch
            device_name = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"
        except ImportError:
            device_name = "unknown"
    topos = ";".join(",".join(f"{a}-{b}" for a, b in np.asarray(t).reshape(-1, 2)) for t, _ in terms)
    dims = ",".join(str(int(d)) for d in evaluator.dims)
    return f"{device_name}|r={evaluator.r}|p={evaluator.p}|dims={dims}|{topos}"


def _time(evaluator, G_dev, S_dev, terms, reps):
    best = np.inf
    for _ in range(reps):
        evaluator.zero_device(S_dev, evaluator.slab)
        evaluator.event_record(6)
        for topo, fac in terms:
            evaluator.compute_self_energy_device(G_dev, topo, float(fac), S_dev)
        evaluator.event_record(7)
        best = min(best, evaluator.event_elapsed(6, 7))
    return best


def tune_sigma(evaluator, G_dev, S_dev, terms, reps=2, params=None, cache_path=None, device_name=None):
    """Tune the launch shapes for ``terms`` (list of (topology, factor)) with G in device buffer ``G_dev``
    (``S_dev`` is scratch for the result).  Leaves the evaluator on the best setting and returns
    (setting, table of (parameter, value, ms))."""
    params = params or list(CANDIDATES)
    _time(evaluator, G_dev, S_dev, terms, 1)  # work lists and edge tables for the current setting
    current = evaluator.get_tuning()
    best_ms = _time(evaluator, G_dev, S_dev, terms, reps)
    table = [("start", dict(current), best_ms)]
    for name in params:
        for value in CANDIDATES[name]:
            if value == current[name]:
                continue
            evaluator.set_tuning(**{name: value})
            _time(evaluator, G_dev, S_dev, terms, 1)
            ms = _time(evaluator, G_dev, S_dev, terms, reps)
            table.append((name, value, ms))
            if ms < best_ms:
                best_ms = ms
                current[name] = value
        evaluator.set_tuning(**current)
    path = cache_path or default_cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache = json.load(open(path)) if os.path.exists(path) else {}
        cache[config_key(evaluator, terms, device_name)] = {"setting": current, "ms": best_ms}
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return current, table


def apply_cached(evaluator, terms, cache_path=None, device_name=None):
    """Apply the recorded setting of this configuration, if any; returns it or None."""
    path = cache_path or default_cache_path()
    if not os.path.exists(path):
        return None
    try:
        entry = json.load(open(path)).get(config_key(evaluator, terms, device_name))
    except (OSError, ValueError):
        return None
    if entry:
        evaluator.set_tuning(**entry["setting"])
        return entry["setting"]
    return None
