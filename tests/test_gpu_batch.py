"""Batched mixed-codec decoding on the GPU: one persistent launch over brle
chunks, RLE v1 / RLE v2 lane streams, LZSS chunks and Deflate streams of
uneven sizes, under the static mapping and the dynamic work queue, bit-exact
against every item's column (whose containers the oracle also decodes)."""
import numpy as np
import pytest

import compression_b200.batch as B
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plan(cuda):
    items = B.make_mixed_batch(7, 120, 48 << 20)
    for it in items:
        rc, out = oracle.decode(it.enc)
        assert rc == 0 and np.array_equal(out, it.raw)
    return B.build_plan(items, cuda)


def test_static_mapping(plan):
    import torch
    plan.d_out.zero_()
    B.launch(plan, None, dynamic=False)
    torch.cuda.synchronize()
    assert B.verify(plan)


def test_dynamic_queue_any_order(plan):
    import torch
    n = plan.tasks.size
    for order in (np.arange(n)[::-1], np.random.default_rng(0).permutation(n)):
        plan.d_out.zero_()
        d_order = torch.from_numpy(order.astype(np.int32)).cuda()
        B.launch(plan, d_order, dynamic=True)
        torch.cuda.synchronize()
        assert B.verify(plan)
    d = B.task_durations_ns(plan)
    assert (d > 0).all()


def test_batch_corrupt_task_reports_and_others_decode(plan, cuda):
    import torch
    # a task whose lane bound is exceeded fails alone; the rest still decode
    bad = plan.tasks.copy()
    i = int(np.nonzero(bad["codec"] == 0)[0][0])  # a brle task
    bad["src_len"][i] = max(1, int(bad["src_len"][i]) // 2)
    d_bad = torch.from_numpy(bad.view(np.uint8).copy()).to(cuda)
    saved = plan.d_tasks
    plan.d_tasks = d_bad
    try:
        plan.d_status.zero_()
        B.launch(plan, None, dynamic=True)
        torch.cuda.synchronize()
        st = plan.d_status.cpu().numpy()
        assert st[i] != 0 and (np.delete(st, i) == 0).all()
    finally:
        plan.d_tasks = saved
