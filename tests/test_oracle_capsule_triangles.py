"""The oracle's capsule-against-triangles restatement, pinned to the reference.

``tests/golden/capsule_triangles.npz`` holds the reference's compiled
``capsule_triangles`` answers (``_collide_native.pyx:454-574``) for hand-placed
floors, walls, ceilings, rims and slivers, seeded random triangles around
tilted capsules, degenerate triangles and grid-mesh candidates. The oracle
must reproduce them bit for bit; the hand-worked cases also carry the known
answers the reference's own batch tests state (depths and normals a capsule a
known distance into a known plane must give).
"""
import numpy as np
import pytest

import pyoracle
from golden_util import GOLDEN

FIX = np.load(GOLDEN + '/capsule_triangles.npz')


def _query(q):
    off = FIX['tri_off']
    s, e = int(off[q]), int(off[q + 1])
    c = FIX['caps'][q]
    return c, s, e


@pytest.mark.parametrize('q', range(len(FIX['caps'])))
def test_oracle_matches_reference_bit_for_bit(q):
    c, s, e = _query(q)
    hit, points, normals, depths = pyoracle.capsule_triangles(c[:3], c[3:6], c[6], FIX['verts'][s:e])
    assert np.array_equal(hit, FIX['hit'][s:e].astype(bool))
    assert np.array_equal(points, FIX['points'][s:e])
    assert np.array_equal(normals, FIX['normals'][s:e])
    assert np.array_equal(depths, FIX['depths'][s:e])


def test_known_answers_of_the_hand_placed_cases():
    """Capsule half height 0.5, radius 0.4 (test_collide_batch.py:38-112)."""
    ans = [pyoracle.capsule_triangles(FIX['caps'][q][:3], FIX['caps'][q][3:6], FIX['caps'][q][6],
                                      FIX['verts'][_query(q)[1]:_query(q)[2]]) for q in range(10)]
    # resting 0.2 into the floor: pushed straight up, contact on the plane; far triangle untouched
    hit, pts, nrm, dep = ans[0]
    assert list(hit) == [True, False, True]
    assert nrm[0] == pytest.approx([0.0, 1.0, 0.0]) and dep[0] == pytest.approx(0.2)
    assert pts[0][1] == pytest.approx(0.0)
    assert not ans[1][0][0]                                          # clear of the floor
    assert ans[2][2][0] == pytest.approx([0.0, -1.0, 0.0])            # driven deep: pushed down
    assert ans[2][3][0] == pytest.approx(0.6)                         # by its whole reach
    assert not ans[3][0][0]                                          # wholly below
    assert ans[4][2][0] == pytest.approx([0.0, -1.0, 0.0]) and ans[4][3][0] == pytest.approx(0.2)
    assert ans[5][2][0] == pytest.approx([-1.0, 0.0, 0.0]) and ans[5][3][0] == pytest.approx(0.15)
    hit, pts, nrm, _ = ans[6]                                         # off the rim, toward the corner
    assert hit[0] and pts[0] == pytest.approx([0.0, 0.0, 0.0])
    assert nrm[0] == pytest.approx([-np.sqrt(0.5), 0.0, -np.sqrt(0.5)], abs=1e-6)
    assert np.all(np.isfinite(ans[7][2]))                            # sliver: never a NaN normal
    assert not ans[9][0].any()                                       # nowhere near


def test_every_branch_is_exercised():
    """Face contacts, rim contacts and misses all occur in the fixture."""
    hit = FIX['hit'].astype(bool)
    n = FIX['normals']
    assert hit.sum() > 500 and (~hit).sum() > 500
    # rim normals are not perpendicular to their triangle's face
    v = FIX['verts']
    face = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    fl = np.linalg.norm(face, axis=1)
    ok = hit & (fl > 1e-9)
    cosang = np.abs(np.einsum('ij,ij->i', n[ok], face[ok]) / fl[ok])
    assert (cosang > 1 - 1e-12).sum() > 100 and (cosang < 0.99).sum() > 100


def test_empty_batch():
    hit, pts, nrm, dep = pyoracle.capsule_triangles(np.zeros(3), np.ones(3), 0.5, np.zeros((0, 3, 3)))
    assert len(hit) == len(pts) == len(nrm) == len(dep) == 0
