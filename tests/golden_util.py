"""Load the committed golden fixtures (made by tests/golden/make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
SCENES = ('pyramid', 'debris', 'convex', 'chain', 'spheres', 'capsules', 'zones', 'terrain', 'ridge', 'conveyor',
          'degenerate', 'rods', 'convex_late')


def load(name):
    with np.load(os.path.join(GOLDEN, name + '.npz')) as z:
        return {k: z[k] for k in z.files}


def checkpoint(data, step):
    """``(inputs, outputs)`` dicts of one checkpoint."""
    pin = 'ck%d/in/' % step
    pout = 'ck%d/out/' % step
    ins = {k[len(pin):]: v for k, v in data.items() if k.startswith(pin)}
    outs = {k[len(pout):]: v for k, v in data.items() if k.startswith(pout)}
    return ins, outs


EVENT_KINDS = ('enter', 'stay', 'exit')


def events_from_overlaps(prev, new):
    """Trigger events of one step as the reference forms them
    (triggers.py:36-42), as a sorted array of (kind code, trigger, other)."""
    ev = [(0,) + p for p in new - prev] + [(1,) + p for p in new & prev] + [(2,) + p for p in prev - new]
    return np.array(sorted(ev), dtype=np.int32).reshape(-1, 3)


def pair_set(arr):
    return {(int(a), int(b)) for a, b in np.asarray(arr).reshape(-1, 2)}


def checkpoints(data):
    return [int(s) for s in data['meta/checkpoints']]
