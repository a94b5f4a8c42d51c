"""The allocation-free sweep-and-prune entry point, through the C ABI.

``omi_sweep_pairs_noalloc`` serves callers that cannot allocate device
memory (a fixed up-front memory pool, a real-time loop where cudaMalloc would
stall the device mid-frame): it works entirely in a fixed scratch array
inside the library and in the caller's own device buffers. This file checks
that it returns exactly the pair list of the arena path (``omi_broadphase``
inside ``omi_step``, read back with ``omi_get_pairs``) for the same AABBs, on
two calls in a row, and that it refuses worlds above its fixed limit. Named
so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200._lib import NOALLOC_MAX_BODIES, OMI_E_ARG, load_library

pytestmark = pytest.mark.gpu


def _noalloc_pairs(world, filter_row=None, filter_matrix=None, rows=0, cap_extra=16):
    import torch
    lib = load_library()
    n = world.body_count
    dev = torch.device('cuda', 0)
    amin = torch.tensor(np.ascontiguousarray(world.aabb_min), dtype=torch.float64, device=dev)
    amax = torch.tensor(np.ascontiguousarray(world.aabb_max), dtype=torch.float64, device=dev)
    mt = torch.tensor(np.asarray(world.motion_type, np.int32), dtype=torch.int32, device=dev)
    fr = fm = None
    if filter_row is not None:
        fr = torch.tensor(np.asarray(filter_row, np.int32), dtype=torch.int32, device=dev)
        fm = torch.tensor(np.asarray(filter_matrix, np.uint8), dtype=torch.uint8, device=dev)
    results = []
    for _ in range(2):                        # two calls in a row share the scratch
        cap = 4 * n + cap_extra
        pairs = torch.full((cap, 2), -7, dtype=torch.int32, device=dev)
        npairs = torch.full((1,), -1, dtype=torch.int32, device=dev)
        err = C.create_string_buffer(256)
        stream = torch.cuda.current_stream(dev)
        rc = lib.omi_sweep_pairs_noalloc(
            amin.data_ptr(), amax.data_ptr(), mt.data_ptr(),
            fr.data_ptr() if fr is not None else None, fm.data_ptr() if fm is not None else None,
            rows, n, pairs.data_ptr(), cap, npairs.data_ptr(), stream.cuda_stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        k = int(npairs.item())
        assert 0 <= k <= cap
        results.append(pairs[:k].cpu().numpy())
    return results


@pytest.mark.parametrize('name,builder,steps', [
    ('debris700', lambda: scenes.debris(n=700, seed=5, extent=9.0, height=10.0, ground=30.0), 90),
    ('pyramid', lambda: scenes.pyramid(), 5),
])
def test_noalloc_matches_arena_broadphase(name, builder, steps):
    w, meta = builder()
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(steps)
    b.sync_to_host()                         # AABBs of the last step's refit
    expected = b.pairs(0)
    assert len(expected) > 0
    for got in _noalloc_pairs(w):
        assert np.array_equal(got, expected), name


def test_noalloc_with_collision_filters():
    w, meta = scenes.feature_mix()
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(30)
    b.sync_to_host()
    expected = b.pairs(0)
    arrays = b.packed.arrays
    rows = int(arrays['w_filter_rows'][0])
    for got in _noalloc_pairs(w, arrays['filter_row'], arrays['filter_matrix'], rows):
        assert np.array_equal(got, expected)


def test_noalloc_refuses_worlds_above_its_limit():
    import torch
    lib = load_library()
    dev = torch.device('cuda', 0)
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    err = C.create_string_buffer(256)
    rc = lib.omi_sweep_pairs_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, None, 0,
                                     NOALLOC_MAX_BODIES + 1, buf.data_ptr(), 1, buf.data_ptr(),
                                     None, err, 256)
    assert rc == OMI_E_ARG
    assert str(NOALLOC_MAX_BODIES) in err.value.decode()
