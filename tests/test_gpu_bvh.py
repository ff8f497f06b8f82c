"""The device BVH builder against the host builder, bit for bit (lux_bvh8_build).

Both run the same binned-SAH binary build (32 bins, SA(L) nL + SA(R) nR, first best split in
axis-then-bin order, stable partitions, the two-primitive and coincident-centroid rules) and the
same collapse and quantisation in the same floating-point order, so the 80-byte nodes, the leaf
order, the roots and the depths must be identical. Cases: random and clustered boxes (runs of
coincident centroids take the positional split), trees of 1, 2, 32, 33 primitives around the
warp-subtree threshold, many trees at once, and the triangle boxes of a 200k-triangle scene."""
import numpy as np
import pytest

import luxion_b200 as lx
from test_bvh_host import NODE, check_tree, random_boxes

pytestmark = pytest.mark.gpu


def same_build(boxes, tb):
    h = lx.bvh8_build(boxes, tb, on_device=False)
    d = lx.bvh8_build(boxes, tb, on_device=True)
    assert np.array_equal(h[2], d[2]), ("roots", h[2][:8], d[2][:8])
    assert np.array_equal(h[3], d[3]), ("depths", h[3][:8], d[3][:8])
    assert h[0].shape == d[0].shape, ("node counts", h[0].shape, d[0].shape)
    bad = np.nonzero(np.any(h[0] != d[0], axis=1))[0]
    if len(bad):
        hn, dn = h[0][bad[0]].view(NODE), d[0][bad[0]].view(NODE)
        raise AssertionError(f"{len(bad)} nodes differ, first {bad[0]}: host {hn} device {dn}")
    bad = np.nonzero(h[1] != d[1])[0]
    assert len(bad) == 0, (f"{len(bad)} leaf records differ, first {bad[:4]}", h[1][bad[:4]], d[1][bad[:4]])
    return d


@pytest.mark.parametrize("sizes,clustered,seed", [
    ([1, 2, 3, 31, 32, 33, 34, 100], False, 1),
    ([5000], False, 2),
    ([5000], True, 3),
    ([70000, 3, 40000, 1, 257], False, 4),
    ([200] * 150, True, 5),
])
def test_device_build_equals_host_build(sizes, clustered, seed):
    tb = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    boxes = random_boxes(int(tb[-1]), seed=seed, clustered=clustered)
    raw, order, roots, depth = same_build(boxes, tb)
    nodes = raw.view(NODE).reshape(-1)
    if sum(sizes) <= 10000:
        for t in range(len(sizes)):
            check_tree(nodes, order, boxes, roots[t], int(tb[t]), int(tb[t + 1]))


def test_device_build_equals_host_build_on_scene_triangles():
    """Triangle boxes of a 200k-triangle instanced scene's meshes, padded as the scene build pads
    them (1e-6 of the coordinate magnitude + 1e-9)."""
    s = lx.random_scene(seed=21, num_instances=40, total_tris=200000, min_tris=2000, max_tris=20000,
                        num_emissive=4, num_textures=1, texture_size=8, env_width=0, env_height=0,
                        width=8, height=8, trace_depth=4)
    d = s.desc
    all_boxes, sizes = [], []
    for m in range(d.num_meshes):
        md = d.meshes[m]
        P = np.ctypeslib.as_array(md.positions, shape=(md.num_verts * 3,)).reshape(-1, 3)
        I = np.ctypeslib.as_array(md.indices, shape=(md.num_tris * 3,)).reshape(-1, 3)
        tri = P[I]
        lo, hi = tri.min(1), tri.max(1)
        pad = (np.float32(1e-6) * np.maximum(np.abs(lo), np.abs(hi))).astype(np.float32) + np.float32(1e-9)
        all_boxes.append(np.concatenate([lo - pad, hi + pad], 1).astype(np.float32))
        sizes.append(md.num_tris)
    tb = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    same_build(np.concatenate(all_boxes), tb)
