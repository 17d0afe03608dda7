"""Known answers of the numpy contact restatement (no GPU): closed-form
primitive contacts whose witness points, normals, margins and counts follow
from the geometry by hand."""

import numpy as np

from oracle import contacts as oc
from sap_warp_b200._abi import SAPB_SHAPE_BOX, SAPB_SHAPE_PLANE, SAPB_SHAPE_SPHERE
from sap_warp_b200.collision import ShapeSet


def _scene(types, scales, poses, X=None):
    """One world: shape i on body i at pose poses[i], then a ground plane."""
    n = len(types)
    Xs = np.zeros((n + 1, 7))
    Xs[:, 6] = 1.0
    if X is not None:
        Xs[:n] = X
    shapes = ShapeSet(num_worlds=1, shapes_per_world=n, num_global_shapes=1,
                      shape_type=np.array(list(types) + [SAPB_SHAPE_PLANE], np.int32),
                      shape_scale=np.array(list(scales) + [[0.0, 0.0, 0.0]], float), shape_X_bs=Xs,
                      shape_body=np.array(list(range(n)) + [-1], np.int32))
    bq = np.zeros((n, 7))
    for i, p in enumerate(poses):
        bq[i, :3] = p[:3]
        bq[i, 3:] = p[3:] if len(p) == 7 else [0, 0, 0, 1]
    return shapes, bq


def test_sphere_on_plane():
    shapes, bq = _scene([SAPB_SHAPE_SPHERE], [[0.1, 0, 0]], [[0.3, -0.2, 0.095]])
    c = oc.generate(shapes, bq, gap=1e-3)
    assert list(c["shape0"]) == [1] and list(c["shape1"]) == [0]
    np.testing.assert_allclose(c["point0"][0], [0.3, -0.2, 0.0])
    np.testing.assert_allclose(c["point1"][0], [0.0, 0.0, 0.0])
    np.testing.assert_allclose(c["normal"][0], [0.0, 0.0, 1.0])
    assert c["margin0"][0] == 0.0 and c["margin1"][0] == 0.1
    phi = np.dot([0.3, -0.2, 0.095] - c["point0"][0], c["normal"][0]) - c["margin0"][0] - c["margin1"][0]
    np.testing.assert_allclose(phi, -0.005)
    # lifted above the gap: no contact
    shapes, bq = _scene([SAPB_SHAPE_SPHERE], [[0.1, 0, 0]], [[0.3, -0.2, 0.1011]])
    assert len(oc.generate(shapes, bq, gap=1e-3)["shape0"]) == 0


def test_thin_box_on_plane_keeps_the_four_deepest_corners():
    """A box 0.2 mm high resting on the ground, tilted slightly: all eight
    corners are within the 1 mm gap and the four bottom ones are kept."""
    h = np.array([0.1, 0.05, 1e-4])
    tilt = 0.0005
    q = np.array([np.sin(tilt / 2), 0, 0, np.cos(tilt / 2)])
    shapes, bq = _scene([SAPB_SHAPE_BOX], [h], [np.concatenate([[0, 0, 2e-4], q])])
    c = oc.generate(shapes, bq, gap=1e-3)
    assert len(c["shape0"]) == 4
    # the kept corners are the bottom face (z = -h) in the box frame
    np.testing.assert_allclose(np.sort(c["point1"][:, 2]), [-h[2]] * 4)
    np.testing.assert_allclose(c["point0"][:, 2], 0.0, atol=1e-15)
    assert np.all(c["normal"] == [0.0, 0.0, 1.0])


def test_overlapping_spheres():
    shapes, bq = _scene([SAPB_SHAPE_SPHERE, SAPB_SHAPE_SPHERE], [[0.1, 0, 0], [0.05, 0, 0]],
                        [[0, 0, 1.0], [0.09, 0.12, 1.0]])
    c = oc.generate(shapes, bq)
    assert list(zip(c["shape0"], c["shape1"])) == [(0, 1)]
    np.testing.assert_allclose(c["normal"][0], [0.6, 0.8, 0.0])
    phi = 0.15 - c["margin0"][0] - c["margin1"][0]
    np.testing.assert_allclose(phi, 0.0, atol=1e-15)


def test_sphere_over_box_face():
    """Sphere above the +z face of a rotated box: normal from the box to the
    sphere along the box's rotated +z, witness point on that face."""
    ang = 0.3
    q = np.array([np.sin(ang / 2), 0, 0, np.cos(ang / 2)])
    up = oc.qrot(q, np.array([0.0, 0.0, 1.0]))
    centre = np.array([0.0, 0.0, 1.0])
    sphere_at = centre + (0.05 + 0.04) * up  # box half height 0.05, radius 0.04: touching
    shapes, bq = _scene([SAPB_SHAPE_BOX, SAPB_SHAPE_SPHERE], [[0.2, 0.2, 0.05], [0.04, 0, 0]],
                        [np.concatenate([centre, q]), sphere_at])
    c = oc.generate(shapes, bq)
    assert list(zip(c["shape0"], c["shape1"])) == [(0, 1)]
    np.testing.assert_allclose(c["normal"][0], up)
    np.testing.assert_allclose(c["point0"][0], [0.0, 0.0, 0.05], atol=1e-15)
    assert c["margin1"][0] == 0.04


def test_small_box_on_big_box():
    """A smaller box centred on a bigger one: its four bottom corners touch
    the top face of the bigger box (normal +z from the lower to the upper);
    the bigger box's corners are outside the smaller one."""
    shapes, bq = _scene([SAPB_SHAPE_BOX, SAPB_SHAPE_BOX], [[0.3, 0.3, 0.1], [0.1, 0.1, 0.1]],
                        [[0, 0, 0.5], [0.02, -0.03, 0.6995]])
    c = oc.generate(shapes, bq)
    assert len(c["shape0"]) == 4
    assert np.all(c["shape0"] == 0) and np.all(c["shape1"] == 1)
    np.testing.assert_allclose(c["normal"], np.tile([0.0, 0.0, 1.0], (4, 1)))
    np.testing.assert_allclose(c["point0"][:, 2], 0.1)
    np.testing.assert_allclose(c["point1"][:, 2], -0.1)
    world1 = bq[1, :3] + c["point1"]
    phi = np.einsum("ij,ij->i", world1 - (bq[0, :3] + c["point0"]), c["normal"])
    np.testing.assert_allclose(phi, -5e-4, atol=1e-12)


def test_crossed_box_edges_touch_edge_to_edge():
    """Two unit cubes each standing on an edge, the lower one's top edge along
    x, the upper one's bottom edge along y, crossing above the origin with
    1 mm of overlap: no corner of either cube is inside the other, so the one
    contact is edge-edge -- normal +z from the lower to the upper cube,
    witness points on the two edges at the crossing, phi0 = -1 mm."""
    r = np.sqrt(0.5)
    qx = np.array([np.sin(np.pi / 8), 0.0, 0.0, np.cos(np.pi / 8)])  # 45 degrees about x
    qy = np.array([0.0, np.sin(np.pi / 8), 0.0, np.cos(np.pi / 8)])  # 45 degrees about y
    top = r  # the lower cube's top edge height
    z1 = top + r - 1e-3
    shapes, bq = _scene([SAPB_SHAPE_BOX, SAPB_SHAPE_BOX], [[0.5, 0.5, 0.5], [0.5, 0.5, 0.5]],
                        [np.concatenate([[0.0, 0.0, 0.0], qx]), np.concatenate([[0.0, 0.0, z1], qy])])
    c = oc.generate(shapes, bq, gap=1e-4)
    edge = [k for k in range(len(c["shape0"])) if c["shape0"][k] == 0 and c["shape1"][k] == 1]
    assert len(edge) == 1, c
    k = edge[0]
    np.testing.assert_allclose(c["normal"][k], [0.0, 0.0, 1.0], atol=1e-12)
    w0 = bq[0, :3] + oc.qrot(bq[0, 3:], c["point0"][k])
    w1 = bq[1, :3] + oc.qrot(bq[1, 3:], c["point1"][k])
    np.testing.assert_allclose(w0, [0.0, 0.0, top], atol=1e-12)
    np.testing.assert_allclose(w1, [0.0, 0.0, z1 - r], atol=1e-12)
    np.testing.assert_allclose(np.dot(w1 - w0, c["normal"][k]), -1e-3, atol=1e-12)
    # lifted 1 mm clear of each other: nothing
    shapes, bq = _scene([SAPB_SHAPE_BOX, SAPB_SHAPE_BOX], [[0.5, 0.5, 0.5], [0.5, 0.5, 0.5]],
                        [np.concatenate([[0.0, 0.0, 0.0], qx]), np.concatenate([[0.0, 0.0, top + r + 1e-3], qy])])
    c = oc.generate(shapes, bq, gap=1e-4)
    assert not any(c["shape0"][k] == 0 and c["shape1"][k] == 1 for k in range(len(c["shape0"])))
