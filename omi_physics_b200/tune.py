"""Autotuner of the step's launch configuration and of the groups per GPU.

Nothing the step computes depends on how its kernels are launched: the
contact sweep is a dataflow whose result is fixed by its dependency graph,
pairs are written at scanned offsets, and every other kernel works per body,
pair or contact. So the launch configuration (``OmiTuning``: warps per
sweep block and how far a block splits for small worlds, block size and
blocks per SM of the pair passes, block size of the analytic narrowphase,
warps per GJK/EPA block) and the number of concurrently stepped groups are
free choices, and the fastest one depends on the GPU and the workload.

:func:`autotune` searches them by coordinate descent: starting from the
defaults, each parameter in turn takes the value with the lowest measured
step time (CUDA events around ``steps`` steps after ``warmup``), the others
held, for ``rounds`` passes; then the group count is searched the same way
with the chosen launch configuration. Results are cached per (GPU name,
workload signature) in a JSON file (``$OMI_TUNING_CACHE``, else
``~/.cache/omi_physics_b200/tuning.json``); the package ships the entries
measured on B200 (``tuned.json`` beside this file), consulted after the user
cache. :func:`lookup` returns a cached entry, which
:class:`~omi_physics_b200.groups.WorldGroups` applies by default.
"""
import json
import math
import os
from typing import Callable, Dict, Optional, Sequence

from ._lib import OmiError

#: values each launch parameter may take, the default first
SPACE = {
    'sweep_warps': (8, 4),
    'sweep_max_split': (4, 2, 1),
    'pair_block': (256, 128, 512),
    'pair_blocks_per_sm': (16, 8, 32),
    'narrow_block': (128, 64, 256),
    'gjk_warps': (4, 2, 8),
    'wide_sweep_blocks': (16, 1, 8, 24, 32, 64, 148),
    'wide_cluster': (16, 8, 0),
    'sweep_claim': (32, 16, 8),
}
#: group counts tried for a many-world workload (a single world is one group)
GROUP_CHOICES = (4, 2, 3, 6)

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED = os.path.join(HERE, 'tuned.json')


def cache_path() -> str:
    return os.environ.get('OMI_TUNING_CACHE') or os.path.join(
        os.path.expanduser('~'), '.cache', 'omi_physics_b200', 'tuning.json')


def signature(worlds: Sequence) -> str:
    """Workload signature: world count, total and largest body counts (each
    rounded to a power of two), and whether hulls / capsules (GJK/EPA) or
    joints are present - what moves the best launch configuration."""
    counts = [int(w.body_count) for w in worlds]
    total, largest = sum(counts), max(counts) if counts else 0

    def p2(x):
        return 0 if x <= 0 else int(round(math.log2(x)))
    gjk = joints = False
    for w in worlds:
        shapes = getattr(w, 'shapes', None) or []
        if any(getattr(s, 'type', None) in ('convex', 'capsule', 'cylinder') for s in shapes):
            gjk = True
        if getattr(w, 'joint_constraints', None):
            joints = True
    return 'w%d-n%d-max%d%s%s' % (p2(len(counts)), p2(total), p2(largest), '-gjk' if gjk else '',
                                  '-joints' if joints else '')


def _read(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(gpu: str, sig: str) -> Optional[dict]:
    """A cached tuning entry (``{'launch': {...}, 'groups': G, 'ms': t}``) or None."""
    for path in (cache_path(), SHIPPED):
        entry = _read(path).get(gpu, {}).get(sig)
        if entry is not None:
            return entry
    return None


def store(gpu: str, sig: str, entry: dict, path: Optional[str] = None) -> None:
    path = path or cache_path()
    data = _read(path)
    data.setdefault(gpu, {})[sig] = entry
    os.makedirs(os.path.dirname(path) or '.', exist_ok=True)
    tmp = path + '.tmp'
    with open(tmp, 'w') as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def coordinate_search(measure: Callable[[dict], float], space: Dict[str, Sequence], start: dict,
                      rounds: int = 2, margin: float = 0.01) -> tuple:
    """Minimise ``measure(cfg)`` one key at a time (the others held), for
    ``rounds`` passes or until a pass changes nothing. A candidate replaces
    the best only when faster by more than ``margin`` (relative), so run to
    run noise does not move the choice. Every configuration is measured once
    (results are memoised). Returns (best cfg, its time, trials)."""
    memo = {}

    def m(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in memo:
            memo[key] = float(measure(dict(cfg)))
        return memo[key]
    best = dict(start)
    best_t = m(best)
    for _ in range(rounds):
        changed = False
        for k, values in space.items():
            for v in values:
                if v == best[k]:
                    continue
                cand = dict(best, **{k: v})
                t = m(cand)
                if t < best_t * (1.0 - margin):
                    best, best_t, changed = cand, t, True
        if not changed:
            break
    return best, best_t, len(memo)


def _time_steps(groups, steps: int, warmup: int) -> float:
    """Device milliseconds per step of every group stepped concurrently."""
    import torch
    groups.step(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    main = torch.cuda.current_stream()
    streams = [torch.cuda.ExternalStream(h) for h in groups.stream_handles]
    e0.record(main)
    for s in streams:
        s.wait_event(e0)
    groups.step_async(steps)
    for s in streams:
        ev = torch.cuda.Event()
        ev.record(s)
        main.wait_event(ev)
    e1.record(main)
    torch.cuda.synchronize()
    groups.sync()
    return e0.elapsed_time(e1) / steps


def autotune(worlds: Sequence, dts: Sequence[float] = None, device: int = 0, steps: int = 10,
             warmup: int = 3, rounds: int = 2, groups: Sequence[int] = None, save: bool = True,
             preroll: int = 0) -> dict:
    """Search the launch configuration and the group count for ``worlds`` on
    ``device`` and cache the result. Every candidate is timed after
    ``preroll`` steps from the worlds' state (the regime the workload runs
    in, e.g. settled piles). The worlds' host columns are not touched (their
    clocks are restored)."""
    import torch
    from .groups import WorldGroups
    times = [w.time for w in worlds]
    dts = list(dts) if dts is not None else [w.fixed_dt for w in worlds]
    choices = tuple(groups) if groups is not None else (GROUP_CHOICES if len(worlds) > 1 else (1,))
    trials = 0
    try:
        g0 = choices[0]
        grp = WorldGroups(worlds, dts=dts, groups=g0, device=device, tuning=None, own_streams=True)
        seen = []
        try:
            grp.step(preroll + warmup)          # into the workload's regime, buffers grown

            def measure_launch(cfg):
                try:
                    grp.set_tuning(cfg)
                except OmiError:                # a choice this GPU cannot run (e.g. a 16-CTA cluster)
                    return float('inf')
                seen.append(_time_steps(grp, steps, warmup))
                return seen[-1]
            start = grp.batches[0].ctx.tuning()  # the library's defaults for this GPU
            launch, ms, n = coordinate_search(measure_launch, SPACE, start, rounds)
            trials += n
        finally:
            grp.close()
        default_ms = seen[0]
        best_g, best_ms = g0, ms
        for g in choices[1:]:
            grp = WorldGroups(worlds, dts=dts, groups=g, device=device, tuning=None, own_streams=True)
            try:
                grp.set_tuning(launch)
                grp.step(preroll + warmup)
                t = _time_steps(grp, steps, warmup)
                trials += 1
            finally:
                grp.close()
            if t < best_ms:
                best_g, best_ms = g, t
    finally:
        for w, t in zip(worlds, times):
            w.time = t
    gpu = torch.cuda.get_device_name(device)
    sig = signature(worlds)
    entry = {'launch': launch, 'groups': best_g, 'ms': best_ms, 'trials': trials,
             'default_ms': default_ms, 'default_groups': g0}
    if save:
        store(gpu, sig, entry)
    return entry


def tuned_for(worlds: Sequence, device: int = 0) -> Optional[dict]:
    """The cached entry for these worlds on this device's GPU, or None."""
    try:
        import torch
        gpu = torch.cuda.get_device_name(device)
    except Exception:
        return None
    return lookup(gpu, signature(worlds))


__all__ = ['SPACE', 'GROUP_CHOICES', 'autotune', 'coordinate_search', 'lookup', 'signature',
           'store', 'tuned_for', 'cache_path']
