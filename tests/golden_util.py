"""Load the committed golden fixtures (made by tests/golden/make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
SCENES = ('pyramid', 'debris', 'convex', 'chain', 'spheres', 'capsules')


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


def checkpoints(data):
    return [int(s) for s in data['meta/checkpoints']]
