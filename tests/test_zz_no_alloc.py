"""The allocation-free sweep-and-prune entry point, through the C ABI.

``omi_sweep_pairs_noalloc`` serves callers that cannot allocate device
memory (a fixed up-front memory pool, a real-time loop where cudaMalloc would
stall the device mid-frame): it works entirely in a fixed scratch array
inside the library and in the caller's own device buffers. This file checks
that it returns exactly the pair list of the arena path (``omi_broadphase``
inside ``omi_step``, read back with ``omi_get_pairs``) and of the oracle for
the same AABBs, on two calls in a row: on small worlds, above 8,192 bodies
(where its sort runs in the array rather than in shared memory) and at its
16,384-body limit; that a pair_cap below the pair count writes only the first
pair_cap pairs but reports the full count; that worlds of 0 and 1 bodies give
no pairs; and that it refuses worlds above its fixed limit. Named so pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from omi_physics_b200 import WorldBatch, scenes
from omi_physics_b200._lib import NOALLOC_MAX_BODIES, OMI_E_ARG, load_library

pytestmark = pytest.mark.gpu


def _noalloc_pairs(world, filter_row=None, filter_matrix=None, rows=0, cap_extra=16, cap=None,
                   full=False):
    """Two calls in a row on the world's AABBs; each result is the written
    pairs (``full``: the whole output buffer and the reported count)."""
    import torch
    lib = load_library()
    n = world.body_count
    dev = torch.device('cuda', 0)
    rows_n = max(n, 1)                        # a world of no bodies still passes valid buffers
    amin = torch.zeros((rows_n, 3), dtype=torch.float64, device=dev)
    amax = torch.zeros((rows_n, 3), dtype=torch.float64, device=dev)
    mt = torch.zeros(rows_n, dtype=torch.int32, device=dev)
    if n:
        amin[:n] = torch.from_numpy(np.ascontiguousarray(world.aabb_min, 'd'))
        amax[:n] = torch.from_numpy(np.ascontiguousarray(world.aabb_max, 'd'))
        mt[:n] = torch.from_numpy(np.asarray(world.motion_type, np.int32))
    fr = fm = None
    if filter_row is not None:
        fr = torch.tensor(np.asarray(filter_row, np.int32), dtype=torch.int32, device=dev)
        fm = torch.tensor(np.asarray(filter_matrix, np.uint8), dtype=torch.uint8, device=dev)
    results = []
    for _ in range(2):                        # two calls in a row share the scratch
        if cap is None:
            cap = 4 * n + cap_extra
        pairs = torch.full((max(cap, 1), 2), -7, dtype=torch.int32, device=dev)
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
        if full:
            results.append((pairs.cpu().numpy(), k))
            continue
        assert 0 <= k <= cap
        results.append(pairs[:k].cpu().numpy())
    return results


def _oracle_pairs(world):
    """The oracle's sweep-and-prune on the world's current AABBs."""
    import pyoracle
    o = pyoracle.OracleWorld.from_world(world)
    n = world.body_count
    o._keep['aabb_min'][:n] = world.aabb_min
    o._keep['aabb_max'][:n] = world.aabb_max
    return o.broadphase()


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


@pytest.mark.parametrize('n', [12000, NOALLOC_MAX_BODIES - 1])
def test_noalloc_large_worlds_match_the_arena_and_the_oracle(n):
    """Above 8,192 bodies the sort keeps its keys in the fixed array, not in
    shared memory; n = 16,383 dynamic bodies plus the ground is the limit."""
    w, meta = scenes.debris(n=n, seed=8, extent=24.0, height=30.0, ground=80.0)
    assert w.body_count == min(n + 1, NOALLOC_MAX_BODIES)
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(40)
    b.sync_to_host()
    expected = b.pairs(0)
    assert len(expected) > 1000
    assert np.array_equal(_oracle_pairs(w), expected)
    for got in _noalloc_pairs(w):
        assert np.array_equal(got, expected)


def test_noalloc_small_pair_cap_writes_only_the_first_pairs():
    w, meta = scenes.debris(n=400, seed=5, extent=7.0, height=8.0, ground=30.0)
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(80)
    b.sync_to_host()
    expected = b.pairs(0)
    assert len(expected) > 40
    for buf, k in _noalloc_pairs(w, cap=25, full=True):
        assert k == len(expected)                  # the full count
        assert np.array_equal(buf[:25], expected[:25])
        assert (buf[25:] == -7).all()              # nothing written past pair_cap


@pytest.mark.parametrize('n_bodies', [0, 1])
def test_noalloc_worlds_of_fewer_than_two_bodies_have_no_pairs(n_bodies):
    api = scenes.default_api()
    m = api.model
    w = api.PhysicsWorld(fixed_dt=1.0 / 60.0)
    if n_bodies:
        w.add_body(m.Motion(type=m.DYNAMIC, mass=1.0), m.Collider(shape=w.add_shape(m.Shape.sphere(0.5))),
                   position=(0.0, 1.0, 0.0))
    for buf, k in _noalloc_pairs(w, cap=4, full=True):
        assert k == 0
        assert (buf == -7).all()


def test_noalloc_matches_the_oracle_on_a_small_world():
    w, meta = scenes.debris(n=700, seed=5, extent=9.0, height=10.0, ground=30.0)
    b = WorldBatch([w], dts=[meta['dt']])
    b.step(90)
    b.sync_to_host()
    want = _oracle_pairs(w)
    for got in _noalloc_pairs(w):
        assert np.array_equal(got, want)
