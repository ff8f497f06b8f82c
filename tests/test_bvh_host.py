"""The host BVH8 builder (lux_bvh8_build with on_device = 0): structural checks on the CPU.

Every box lands in exactly one leaf slot, internal children are contiguous at child_base in
slot order, leaf records are tri_base + rank among the node's leaf slots, and every quantised
slot box contains the boxes below it (the outward rounding the traversal relies on). The device
builder is checked against this one bit for bit on the GPU (tests/test_gpu_bvh.py)."""
import numpy as np
import pytest

import luxion_b200 as lx

NODE = np.dtype([("p", "<f4", 3), ("e", "u1", 3), ("imask", "u1"), ("child_base", "<u4"), ("tri_base", "<u4"),
                 ("meta", "u1", 8), ("qlo", "u1", (3, 8)), ("qhi", "u1", (3, 8))])


def random_boxes(n, seed, clustered=False):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, 3)) * (0.1 if clustered else 10.0)
    if clustered:
        c[: n // 3] = c[0]          # a run of coincident centroids
    h = rng.uniform(0.001, 0.5, (n, 3))
    return np.concatenate([c - h, c + h], 1).astype(np.float32)


def check_tree(nodes, order, boxes, root, t0, t1):
    seen = np.zeros(t1 - t0, np.int64)

    def slot_box(nd, s):
        sc = np.ldexp(1.0, nd["e"].astype(np.int64) - 127)
        return nd["p"] + nd["qlo"][:, s] * sc, nd["p"] + nd["qhi"][:, s] * sc

    def visit(i):
        nd = nodes[i]
        leaves = []
        internal = 0
        rank = 0
        for s in range(8):
            lo, hi = slot_box(nd, s)
            if (nd["meta"][0] >> s) & 1:
                rec = int(nd["tri_base"]) + rank
                rank += 1
                b = int(order[t0 + rec])
                assert t0 <= b < t1
                seen[b - t0] += 1
                sub = [b]
            elif (nd["imask"] >> s) & 1:
                sub = visit(int(nd["child_base"]) + internal)
                internal += 1
            else:
                continue
            bb = boxes[sub]
            assert np.all(lo <= bb[:, :3].min(0)) and np.all(hi >= bb[:, 3:].max(0))
            leaves += sub
        return leaves

    visit(int(root))
    assert np.all(seen == 1)


@pytest.mark.parametrize("sizes,clustered", [([1, 2, 3, 33, 500], False), ([2000], True), ([40, 7, 1, 64], True)])
def test_host_builder_structure(sizes, clustered):
    tb = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    boxes = random_boxes(int(tb[-1]), seed=len(sizes), clustered=clustered)
    raw, order, roots, depth = lx.bvh8_build(boxes, tb, on_device=False)
    nodes = raw.view(NODE).reshape(-1)
    for t in range(len(sizes)):
        check_tree(nodes, order, boxes, roots[t], int(tb[t]), int(tb[t + 1]))
        assert depth[t] >= 1
