"""The rule behind EPA's parallel polytope rebuild, checked against the
reference's dictionary walk on random polytopes (no GPU).

``_rebuild`` (the reference's gjk.py:197-217) walks the faces that see the
new point in order; each edge of a visible face deletes its reverse from an
insertion-ordered dict when present, else is inserted, and the surviving
edges in insertion order make the new faces. The device's lanes use the rule
that, when no directed edge occurs twice among the visible faces, an edge
survives exactly when its reverse is not among them, in walk order - and
fall back to the walk when a directed edge does occur twice. This restates
both in Python: the rule agrees with the walk on closed triangulated
polytopes (convex hulls of random points, every new point outside), and the
duplicate test fires on the degenerate face lists where it could differ.
"""
import numpy as np
import pytest

scipy_spatial = pytest.importorskip('scipy.spatial')


def dict_walk(faces, visible):
    """The reference's _rebuild order: kept faces, then surviving horizon edges."""
    edges = {}
    kept = []
    for f, vis in zip(faces, visible):
        if vis:
            for e in ((f[0], f[1]), (f[1], f[2]), (f[2], f[0])):
                if (e[1], e[0]) in edges:
                    del edges[(e[1], e[0])]
                else:
                    edges[e] = True
        else:
            kept.append(tuple(f))
    return kept, list(edges)


def lane_rule(faces, visible):
    """The device's parallel rule, or None when a directed edge occurs twice
    among the visible faces (the device then runs the walk)."""
    vis_edges = [e for f, v in zip(faces, visible) if v
                 for e in ((f[0], f[1]), (f[1], f[2]), (f[2], f[0]))]
    if len(set(vis_edges)) != len(vis_edges):
        return None
    seen = set(vis_edges)
    kept = [tuple(f) for f, v in zip(faces, visible) if not v]
    return kept, [e for e in vis_edges if (e[1], e[0]) not in seen]


def outward_faces(pts):
    hull = scipy_spatial.ConvexHull(pts)
    faces = []
    c = pts.mean(axis=0)
    for tri in hull.simplices:
        a, b, d = pts[tri]
        if np.dot(np.cross(b - a, d - a), a - c) < 0:
            tri = tri[[0, 2, 1]]
        faces.append(tuple(int(i) for i in tri))
    return faces


@pytest.mark.parametrize('seed', range(40))
def test_rule_equals_the_walk_on_closed_polytopes(seed):
    rng = np.random.default_rng(seed)
    pts = rng.normal(size=(int(rng.integers(6, 40)), 3))
    faces = outward_faces(pts)
    rng.shuffle(faces)                         # the walk's face order is arbitrary on the device too
    for _ in range(5):
        w = rng.normal(size=3) * rng.uniform(1.5, 4.0)
        visible = [np.dot(np.cross(pts[f[1]] - pts[f[0]], pts[f[2]] - pts[f[0]]), w - pts[f[0]]) > 0
                   for f in faces]
        got = lane_rule(faces, visible)
        assert got is not None                 # a closed polytope never repeats a directed edge
        assert got == dict_walk(faces, visible)


def test_repeated_directed_edges_are_detected():
    # two copies of one face: every edge appears twice; the walk then keeps edges the rule would drop
    faces = [(0, 1, 2), (0, 1, 2), (1, 0, 3)]
    visible = [True, True, True]
    assert lane_rule(faces, visible) is None
    kept, edges = dict_walk(faces, visible)
    assert kept == [] and len(edges) > 0
