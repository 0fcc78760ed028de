"""st_build_lbvh_noalloc (static device scratch, no allocation) against st_build_bvh(ST_BVH_LBVH30)
through the C ABI: two builds in a row, each bit-identical to the allocating entry point."""
import ctypes as C

import numpy as np
import pytest

from slimtracin_b200 import api, structs as S

pytestmark = pytest.mark.gpu

MAX_ITEMS = 65536          # ST_NOALLOC_LBVH_MAX_ITEMS


def _boxes(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-40, 40, (n, 3))
    e = rng.uniform(0.01, 2, (n, 3))
    b = np.concatenate([c - e, c + e], 1).astype(np.float32)
    b[n // 2:n // 2 + min(8, n // 2)] = b[0]          # equal codes, ordered by index
    return b


def _noalloc(r, boxes, max_leaf):
    import torch
    n = len(boxes)
    d_boxes = torch.from_numpy(boxes).cuda()
    d_codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_order = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_nodes = torch.zeros(2 * n * S.BVHNODE_DT.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    info = (C.c_uint32 * 2)()
    status = r.L.st_build_lbvh_noalloc(r.ctx, d_boxes.data_ptr(), n, max_leaf, d_codes.data_ptr(),
                                       d_order.data_ptr(), d_nodes.data_ptr(), info, None)
    r._check(status, "st_build_lbvh_noalloc")
    count = int(info[0])
    nodes = d_nodes.cpu().numpy().view(S.BVHNODE_DT)[:count]
    return (d_codes.cpu().numpy().view(np.uint32), d_order.cpu().numpy().view(np.uint32), nodes, count,
            int(info[1]))


def test_noalloc_lbvh_equals_allocating_build_twice_in_a_row(renderer):
    # a large build, then a small one over the same static scratch: stale words from the first
    # must not reach the second
    for n, max_leaf, seed in ((MAX_ITEMS, 2, 5), (777, 4, 6)):
        boxes = _boxes(n, seed)
        codes, order, nodes, count, height = _noalloc(renderer, boxes, max_leaf)
        rc, ro, rn, rcount, rheight = renderer.build_lbvh(boxes, max_leaf, api.ST_BVH_LBVH30)
        assert (count, height) == (rcount, rheight)
        assert np.array_equal(codes, rc)
        assert np.array_equal(order, ro)
        assert np.array_equal(nodes.view(np.uint8), rn.view(np.uint8))


def test_noalloc_lbvh_allocates_nothing():
    """A fresh context (its pooled builder scratch never reserved): after a warm-up call has loaded the
    module, a second call leaves the context's device bytes and the device's free memory unchanged."""
    import torch
    n, max_leaf = 20000, 2
    boxes = _boxes(n, 11)
    d_boxes = torch.from_numpy(boxes).cuda()
    d_codes = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_order = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_nodes = torch.zeros(2 * n * S.BVHNODE_DT.itemsize, dtype=torch.uint8, device="cuda")
    info = (C.c_uint32 * 2)()
    with api.Renderer(device=0) as r:
        def call():
            r._check(r.L.st_build_lbvh_noalloc(r.ctx, d_boxes.data_ptr(), n, max_leaf, d_codes.data_ptr(),
                                               d_order.data_ptr(), d_nodes.data_ptr(), info, None),
                     "st_build_lbvh_noalloc")
        call()
        torch.cuda.synchronize()
        in_use, free = int(r.L.st_device_bytes_in_use(r.ctx)), torch.cuda.mem_get_info()[0]
        first = d_nodes.cpu().numpy().copy()
        d_nodes.zero_()
        torch.cuda.synchronize()
        call()
        torch.cuda.synchronize()
        assert int(r.L.st_device_bytes_in_use(r.ctx)) == in_use
        assert torch.cuda.mem_get_info()[0] == free
        assert np.array_equal(d_nodes.cpu().numpy(), first)


def test_noalloc_lbvh_refuses_more_than_its_scratch(renderer):
    import torch
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    info = (C.c_uint32 * 2)()
    # rejected on the size alone, on the host, before any work is queued
    status = renderer.L.st_build_lbvh_noalloc(renderer.ctx, buf.data_ptr(), MAX_ITEMS + 1, 2, None, buf.data_ptr(),
                                              buf.data_ptr(), info, None)
    assert status == 1     # ST_ERR_INVALID_ARG
