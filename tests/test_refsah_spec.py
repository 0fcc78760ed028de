"""The level-parallel form of the reference's SAH builder that ST_BVH_REF_SAH runs on the device
(slimtracin_b200/csrc/st_refsah.cu), restated in Python float32 and checked against the oracle's
updateSceneBVH (itself pinned to the reference's builder).

The reference builds depth first from an explicit stack, right child first
(builder_top_down.h:229-262).  The device splits a whole tree level at a time, then numbers nodes
and leaf slots from the tree's shape: the children of the k-th split (in right-first depth-first
order) get node ids 1 + 2k and 2 + 2k, leaves take slots in that order, and a node's depth field is
its stack index (a right child's is its parent's + 1).  This test shows that this numbering, applied
to splits made level by level, reproduces the reference's arrays byte for byte."""
import ctypes as C

import numpy as np
import pytest

import oracle
from slimtracin_b200 import scenes, structs as S
from tests import helpers as H

F = np.float32


def _sort(ids, keys):
    """sortNodesByAxis (:92) with partitionNodesByAxis (:66): Lomuto, pivot last, explicit stack."""
    m = len(ids)
    if all(keys[i - 1] < keys[i] for i in range(1, m)):
        return                            # strictly increasing: every partition keeps the order
    stack = [0, m - 1]
    while stack:
        end = stack.pop()
        start = stack.pop()
        pivot, p = keys[end], start
        for i in range(start, end):
            if keys[i] < pivot:
                ids[i], ids[p] = ids[p], ids[i]
                keys[i], keys[p] = keys[p], keys[i]
                p += 1
        ids[end], ids[p] = ids[p], ids[end]
        keys[end], keys[p] = keys[p], keys[end]
        if p - 1 > start:
            stack += [start, p - 1]
        if p + 1 < end:
            stack += [p + 1, end]


def _merge(a, b):                         # mergeAABBs AABB.h:25
    return [a[k] if a[k] < b[k] else b[k] for k in range(3)] + [a[k] if a[k] > b[k] else b[k] for k in range(3, 6)]


def _half(a):                             # getSurfaceAreaOfAABB AABB.h:39
    ex, ey, ez = F(a[3] - a[0]), F(a[4] - a[1]), F(a[5] - a[2])
    return F(F(F(ex * ey) + F(ey * ez)) + F(ez * ex))


def _split(B, ids):
    """splitBVHNode (:168) over one node's items: (left count, the chosen axis' order, child boxes)."""
    m = len(ids)
    best_axis = None
    for a in range(3):
        sid = list(ids)
        keys = [B[i][3 + a] for i in sid]
        _sort(sid, keys)
        L, R = list(B[sid[0]]), list(B[sid[m - 1]])
        lsa, rsa = [None] * m, [None] * m
        for li in range(m):
            ri = m - 1 - li
            if li:
                L, R = _merge(L, B[sid[li]]), _merge(R, B[sid[ri]])
            lsa[li], rsa[ri] = _half(L), _half(R)
        best, lc = F(np.inf), 1
        for ci in range(m - 1):
            cost = F(F(lsa[ci] * F(ci + 1)) + F(rsa[ci + 1] * F(m - 1 - ci)))
            if best > cost:
                best, lc = cost, ci + 1
        if best_axis is None or best < best_axis[0]:
            best_axis = (best, lc, sid)
    _, lc, sid = best_axis
    L, R = list(B[sid[0]]), list(B[sid[m - 1]])
    for i in range(1, lc):
        L = _merge(L, B[sid[i]])
    for i in range(m - 2, lc - 1, -1):
        R = _merge(R, B[sid[i]])
    return lc, sid, L, R


def ref_sah_level_parallel(boxes, max_leaf):
    """buildBVH (:204) the way st_refsah.cu runs it: (nodes, leaf_ids, node_count, height)."""
    n = len(boxes)
    B = [[F(v) for v in b] for b in boxes]
    ids = list(range(n))
    nodes = np.zeros(2 * n, dtype=S.BVHNODE_DT)
    leaf = np.zeros(n, np.uint32)
    if n <= max_leaf:
        box = [F(np.inf)] * 3 + [F(-np.inf)] * 3
        for i in range(n):
            box = _merge(box, B[i])
        nodes[0:1].view(np.float32)[:6] = box
        nodes["child_count"][0] = n
        leaf[:] = np.arange(n)
        return nodes[:1], leaf, 1, 1
    tasks = [dict(start=0, end=n, box=None, split=False)]
    level = [0]
    while level:                          # one tree level at a time
        nxt = []
        for ti in level:
            T = tasks[ti]
            if T["end"] - T["start"] <= max_leaf:
                continue
            lc, sid, L, R = _split(B, ids[T["start"]:T["end"]])
            ids[T["start"]:T["end"]] = sid
            T.update(split=True, left=len(tasks), right=len(tasks) + 1)
            tasks.append(dict(start=T["start"], end=T["start"] + lc, box=L, split=False))
            tasks.append(dict(start=T["start"] + lc, end=T["end"], box=R, split=False))
            nxt += [T["left"], T["right"]]
        level = nxt
    nt = len(tasks)
    internal = [0] * nt                   # internal nodes per subtree (children follow parents)
    for i in reversed(range(nt)):
        if tasks[i]["split"]:
            internal[i] = 1 + internal[tasks[i]["left"]] + internal[tasks[i]["right"]]
    rank, slot, sidx, node = [0] * nt, [0] * nt, [0] * nt, [0] * nt
    height = splits = 0
    for i, T in enumerate(tasks):
        if not T["split"]:
            continue
        splits += 1
        l, r = T["left"], T["right"]
        rank[r], rank[l] = rank[i] + 1, rank[i] + 1 + internal[r]        # right subtree split first
        slot[r], slot[l] = slot[i], slot[i] + tasks[r]["end"] - tasks[r]["start"]
        sidx[r], sidx[l] = sidx[i] + 1, sidx[i]
        node[l], node[r] = 1 + 2 * rank[i], 2 + 2 * rank[i]
        height = max(height, sidx[r])
    for i, T in enumerate(tasks):
        k = node[i]
        if i:
            nodes[k:k + 1].view(np.float32)[:6] = T["box"]
        if T["split"]:
            nodes["first_child_id"][k] = 1 + 2 * rank[i]
            nodes["depth"][node[T["left"]]] = nodes["depth"][node[T["right"]]] = sidx[i]
        else:
            cnt = T["end"] - T["start"]
            nodes["first_child_id"][k], nodes["child_count"][k] = slot[i], cnt
            leaf[slot[i]:slot[i] + cnt] = ids[T["start"]:T["end"]]
    for i, T in enumerate(tasks):
        if i and not T["split"]:
            nodes["depth"][node[i]] = sidx[i]
    nodes["depth"][0] = 0
    nodes[0:1].view(np.float32)[:6] = _merge(list(nodes[1:2].view(np.float32)[:6]), list(nodes[2:3].view(np.float32)[:6]))
    return nodes[:1 + 2 * splits], leaf, 1 + 2 * splits, max(height, 1)


@pytest.mark.parametrize("count,equal_keys", [(1, False), (2, False), (3, False), (16, False), (17, False),
                                              (64, False), (300, True), (1024, False), (4096, False)])
def test_level_parallel_ref_sah_equals_update_scene_bvh(count, equal_keys):
    sd, _ = scenes.moving_scene(seed_offset=count, count=count)
    if equal_keys:
        sd.primitives["position"][::7] = sd.primitives["position"][0]
    sc, keep = sd.to_ctypes()
    boxes = np.zeros((count, 6), np.float32)
    oracle.restatement().orc_primitive_aabbs(C.byref(sc), boxes.ctypes.data)
    ref = sd.copy()
    H.tlas_sah(ref, "orc")
    nodes, leaf, node_count, height = ref_sah_level_parallel(boxes.tolist(), 2)
    assert (node_count, height) == (ref.tlas_node_count, ref.tlas_height)
    assert nodes.tobytes() == ref.tlas_nodes[:node_count].tobytes()
    assert np.array_equal(leaf, ref.tlas_leaf_ids[:count])
