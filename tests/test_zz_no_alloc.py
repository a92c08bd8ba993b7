"""gd_batch_decode_lpt_noalloc (the batch decoder whose order array, sort
buckets and work-queue counter live in a fixed device array of the library)
against gd_batch_decode with caller-provided scratch, on the same batch, two
calls in a row.  Collected last so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

import compression_b200.batch as B
from compression_b200._lib import lib

pytestmark = pytest.mark.gpu

MAX_TASKS = 65536


def test_noalloc_matches_batch_decode(cuda):
    import torch
    items = B.make_mixed_batch(17, 150, 24 << 20)
    plan = B.build_plan(items, cuda)
    n = plan.tasks.size
    assert n <= MAX_TASKS
    # reference run: the existing entry point, identity order, caller scratch
    plan.d_out.zero_()
    plan.d_status.fill_(0xFF)
    B.launch(plan, None, dynamic=True, timing=False)
    torch.cuda.synchronize()
    want_out = plan.d_out.cpu().numpy().copy()
    want_st = plan.d_status.cpu().numpy().copy()
    assert (want_st == 0).all() and B.verify(plan)
    # costs: decompressed bytes per task (any estimate is valid)
    cost = torch.from_numpy(plan.tasks["dst_len"].astype(np.float32)).cuda()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())
    for _ in range(2):
        plan.d_out.zero_()
        plan.d_status.fill_(0xFF)
        rc = lib().gd_batch_decode_lpt_noalloc(p(plan.d_tasks), n, p(cost), plan.max_lane, 0, p(plan.d_status), s)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(plan.d_status.cpu().numpy(), want_st)
        assert np.array_equal(plan.d_out.cpu().numpy(), want_out)
    # non-finite costs: +inf runs first, NaN and -inf last, and the finite
    # costs still set the bucket range; the output is the same either way
    rng = np.random.default_rng(5)
    c = plan.tasks["dst_len"].astype(np.float32)
    for special in ([np.inf], [np.nan], [-np.inf], [np.inf, -np.inf, np.nan]):
        cc = c.copy()
        pick = rng.choice(n, size=max(1, n // 7), replace=False)
        cc[pick] = rng.choice(np.array(special, np.float32), size=pick.size)
        for costs in (cc, np.full(n, special[0], np.float32)):
            cost2 = torch.from_numpy(costs).cuda()
            plan.d_out.zero_()
            plan.d_status.fill_(0xFF)
            rc = lib().gd_batch_decode_lpt_noalloc(p(plan.d_tasks), n, p(cost2), plan.max_lane, 0,
                                                   p(plan.d_status), s)
            assert rc == 0
            torch.cuda.synchronize()
            assert np.array_equal(plan.d_status.cpu().numpy(), want_st), special
            assert np.array_equal(plan.d_out.cpu().numpy(), want_out), special
    # more tasks than the fixed array holds: rejected before any launch
    rc = lib().gd_batch_decode_lpt_noalloc(p(plan.d_tasks), MAX_TASKS + 1, p(cost), plan.max_lane, 0,
                                           p(plan.d_status), s)
    assert rc == 1
