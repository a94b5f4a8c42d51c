"""Serving host logic without a GPU: slot classes, admission policy and the
capacities a packed world needs."""
import pytest

from omi_physics_b200 import scenes
from omi_physics_b200.arena import pack_worlds
from omi_physics_b200.serving import SlotClass, SlotPool, fits, need_of, size_classes


def caps(b, **kw):
    return SlotClass(bodies=b, count=1, **kw).caps()


def test_size_classes_cover_range():
    cl = size_classes(2048, per_class=5)
    assert [c.bodies for c in cl] == [33, 65, 129, 257, 513, 1025, 2049]
    assert all(c.count == 5 for c in cl)


def test_pool_takes_smallest_fitting_and_spills_up():
    pool = SlotPool([caps(65), caps(33), caps(129), caps(33)])
    need = (20, 20, 20, 0, 0, 2, 0)
    a = pool.take(need)
    b = pool.take(need)
    assert {a, b} == {1, 3}                  # both 33-body slots first
    c = pool.take(need)
    assert c == 0                            # then the 65-body slot
    assert pool.take((100, 1, 1, 0, 0, 1, 0)) == 2
    assert pool.take(need) is None           # full: the request waits
    pool.give_back(1)
    assert pool.take(need) == 1
    with pytest.raises(ValueError):
        pool.give_back(0) or pool.give_back(0)


def test_pool_checks_every_capacity():
    pool = SlotPool([caps(64, joints=0), caps(64, joints=8)])
    assert pool.take((10, 10, 10, 0, 4, 1, 0)) == 1
    assert pool.take((10, 10, 10, 0, 4, 1, 0)) is None
    assert not pool.could_ever_fit((10, 10, 10, 0, 9, 1, 0))
    assert pool.could_ever_fit((64, 64, 64, 0, 0, 8, 16))


def test_need_of_packed_serving_world():
    req = scenes.serving_requests(4, seed=5)[2]
    w, meta = scenes.serving_world(req)
    p = pack_worlds([w], [meta['dt']])
    need = need_of(p.scene)
    assert need[0] == w.body_count == req['bodies'] + 1
    assert need[4] == 0
    cl = size_classes(2048, per_class=1)
    assert any(fits(c.caps(), need) for c in cl)
    smallest = min((c for c in cl if fits(c.caps(), need)), key=lambda c: c.bodies)
    assert smallest.bodies >= need[0] and smallest.bodies < 2 * need[0] + 2


def test_pool_grows_by_appended_slots():
    pool = SlotPool([caps(33)])
    need = (20, 20, 20, 0, 0, 2, 0)
    assert pool.take(need) == 0
    assert pool.take(need) is None           # the class is full
    ids = pool.add([caps(33), caps(65)])     # a new chunk of slots
    assert ids == [1, 2]
    assert pool.take(need) == 1              # the new 33-body slot first
    assert pool.take(need) == 2
    pool.give_back(0)
    assert pool.take(need) == 0
    with pytest.raises(ValueError):
        pool.add([caps(33)], first=7)        # ids stay contiguous
