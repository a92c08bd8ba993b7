"""Learned cost model on the GPU: the hand-written backward kernel against
the CPU oracle (tolerance: rel 1e-3 of the gradient's scale, FP32 vs FP64),
training on self-measured task times, and the scheduling gain of
longest-predicted-first over the static mapping."""
import numpy as np
import pytest

import compression_b200.batch as B
from compression_b200.costmodel import CostModel, GraphSchedule, lpt_order, measure_tasks, task_groups
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def test_gradient_matches_oracle(cuda):
    import torch
    rng = np.random.default_rng(1)
    m = CostModel(seed=3)
    X = rng.normal(0, 1, (200, 16)).astype(np.float32)
    y = rng.normal(0, 1, 200).astype(np.float32)
    d_x = torch.from_numpy(X).cuda()
    d_y = torch.from_numpy(y).cuda()
    idx = torch.arange(200, dtype=torch.int32, device="cuda")
    g, loss = m.grad(d_x, d_y, idx, 200)
    p = m.params.cpu().numpy().astype(np.float64)
    ref = mlp_ref.grad(p, X.astype(np.float64), y.astype(np.float64))
    gg = g.cpu().numpy()
    scale = np.abs(ref).max()
    assert np.abs(gg - ref).max() <= 1e-3 * scale
    assert abs(loss.item() - mlp_ref.loss(p, X, y)) <= 1e-4 * max(1.0, mlp_ref.loss(p, X, y))
    # inference kernel against the oracle's forward pass
    pred = m.predict(X * m.sd + m.mu)  # predict() normalises; undo to feed X itself
    ref_o, _ = mlp_ref.forward(p, X.astype(np.float64))
    assert np.allclose(pred - m.y_mu, ref_o, rtol=1e-4, atol=1e-4)


def test_training_learns_a_function(cuda):
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (4000, 16)).astype(np.float32)
    X[:, 15] = 1.0
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] + np.abs(X[:, 3])).astype(np.float32)
    m = CostModel(seed=0)
    losses = m.train(X, y, epochs=30, batch=256, lr=3e-3)
    assert losses[-1] < 0.2 * losses[0]


@pytest.fixture(scope="module")
def batch(cuda):
    # many items of moderate size: the total work per warp, not one long
    # task, sets the makespan, which is where placement matters
    items = B.make_mixed_batch(11, 2400, 480 << 20, 4096, 512 << 10)
    return B.build_plan(items, cuda)


def test_learned_lpt_beats_static_mapping(batch):
    import torch
    plan = batch
    X = B.task_features(plan)
    # self-measured training data: two randomly ordered runs of this batch
    # shape and one of a different batch
    ys = [np.log(np.maximum(measure_tasks(plan, seed=s), 1.0)) for s in (0, 1)]
    m = CostModel(seed=0)
    m.train(np.concatenate([X, X]), np.concatenate(ys), epochs=25, lr=3e-3)
    pred = m.predict(X)
    r = np.corrcoef(pred, ys[0])[0, 1]
    static = B.makespan_ms(plan, None, dynamic=False, reps=5)
    queue = B.makespan_ms(plan, None, dynamic=True, reps=5)
    groups, codec = task_groups(plan), plan.tasks["codec"]
    order = lpt_order(m.predict32(X), groups, codec)  # the scheduler's order: grouped, banded
    learned = B.makespan_ms(plan, order, dynamic=True, reps=5)
    print(f"\ncorr(pred, measured)={r:.3f}  static={static:.3f} ms  queue={queue:.3f} ms  "
          f"learned-LPT={learned:.3f} ms  gain vs static={(1 - learned / static) * 100:.1f}%")
    assert r > 0.8
    assert learned < 0.8 * static  # >= 20% shorter makespan than the static mapping
    plan.d_out.zero_()
    B.launch(plan, order, dynamic=True)
    torch.cuda.synchronize()
    assert B.verify(plan)


def test_graph_captured_schedule(batch):
    import torch
    plan = batch
    X = B.task_features(plan)
    m = CostModel(seed=5)
    m.fit_normaliser(X, np.zeros(X.shape[0]))
    g = GraphSchedule(plan, m, X)
    plan.d_out.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert B.verify(plan)
    # the graph's order (group maximum and stable sort on the device) is the
    # host's grouped longest-first order of the same predictions
    from compression_b200.costmodel import lpt_order_host
    pred = g.d_pred[:plan.tasks.size].cpu().numpy() + np.float32(m.y_mu)
    groups = task_groups(plan)
    assert np.array_equal(g.order.cpu().numpy(), lpt_order_host(pred, groups, plan.tasks["codec"]))
    g2 = GraphSchedule(plan, m, X, banded=False)
    g2.replay()  # the captured order is written when the graph runs
    torch.cuda.synchronize()
    assert np.array_equal(g2.order.cpu().numpy(), lpt_order_host(pred, groups))
    # every RLE chunk's 32 lane tasks sit together in it
    pos = np.empty(plan.tasks.size, np.int64)
    pos[g.order.cpu().numpy()] = np.arange(plan.tasks.size)
    for gid in np.unique(groups[np.isin(plan.tasks["codec"], (1, 2))])[:50]:
        p = np.sort(pos[groups == gid])
        assert p[-1] - p[0] == p.size - 1


# ---------------------------------------------------------------------------
# header features on the device (gd_task_features) against a host walk of the
# same headers
# ---------------------------------------------------------------------------

_W = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 26, 28, 30, 32, 40,
      48, 56, 64]


def _cfb(b):
    for w in [1] + list(range(2, 25)) + [26, 28, 30, 32, 40, 48, 56, 64]:
        if b <= w:
            return w
    return 64


def _walk_rlev1(s):
    pos, hdr, lit, vals = 0, 0, 0, 0
    while pos < len(s):
        h = s[pos] - 256 if s[pos] > 127 else s[pos]
        pos += 1
        hdr += 1
        if h < 0:
            nv, lit, vals = -h, lit - h, vals - h
        else:
            nv, vals = 1, vals + h + 3
            pos += 1
        for _ in range(nv):
            while pos < len(s) and s[pos] & 0x80:
                pos += 1
            pos += 1
    return hdr, (lit / vals if vals else 0.0)


def _walk_rlev2(s):
    pos, runs, unpack = 0, 0, 0
    while pos < len(s):
        h = s[pos]
        k = h >> 6
        runs += 1
        if k == 0:
            pos += 2 + ((h >> 3) & 7)
            continue
        n, fbw = (((h & 1) << 8) | s[pos + 1]) + 1, _W[(h >> 1) & 31]
        if k == 1:
            unpack += 1
            pos += 2 + (n * fbw + 7) // 8
        elif k == 2:
            unpack += 1
            b2, b3 = s[pos + 2], s[pos + 3]
            pos += 4 + (b2 >> 5) + 1 + (n * fbw + 7) // 8 + ((b3 & 31) * _cfb(_W[b2 & 31] + (b3 >> 5) + 1) + 7) // 8
        else:
            q = pos + 2
            for _ in range(2):
                while s[q] & 0x80:
                    q += 1
                q += 1
            pos = q + (((n - 2) * fbw + 7) // 8 if (h >> 1) & 31 else 0)
    return runs, (unpack / runs if runs else 0.0)


def _walk_lzss(cols):
    toks = lits = 0
    for s in cols:
        pos, k, head = 0, 8, 0
        while pos < len(s):
            if k == 8:
                head, k, pos = s[pos], 0, pos + 1
                continue
            lit = (head >> k) & 1
            k += 1
            toks += 1
            lits += lit
            pos += 1 if lit else 2
    return toks, (lits / toks if toks else 0.0)


def test_header_features_match_host_walk(cuda):
    import oracle
    items = B.make_mixed_batch(23, 60, 12 << 20, 4096, 1 << 20)
    plan = B.build_plan(items, cuda)
    H = B.header_features(plan)
    T = plan.tasks
    lanes = {}
    for ti in range(T.size):
        it = plan.items[plan.task_item[ti]]
        e, k = it.enc, int(plan.extra["task_chunk"][ti])
        units, share, dens = 0, 0.0, 0.0
        out_b = float(T["dst_len"][ti])
        if it.codec == "brle":
            p = e.meta["ptr"]
            s = e.data[int(p[k]):int(p[k + 1])].tolist()
            pos = lit = 0
            while pos < len(s):
                units += 1
                if s[pos] > 127:
                    lit += 1
                    pos += s[pos] - 126
                else:
                    pos += 2
            share, dens = (lit / units if units else 0.0), units * 1024 / out_b
        elif it.codec in ("rlev1", "rlev2", "lzss"):
            if plan.task_item[ti] not in lanes:
                lanes[plan.task_item[ti]] = oracle.export_lanes(e)
            L, off = lanes[plan.task_item[ti]]
            if it.codec == "lzss":
                cols = [L[off[32 * k + r]:off[32 * k + r + 1]].tolist() for r in range(32)]
                units, share = _walk_lzss(cols)
                dens = units * 1024 / out_b
            else:
                t = int(T["lane"][ti])
                s = L[off[32 * k + t]:off[32 * k + t + 1]].tolist()
                units, share = (_walk_rlev1 if it.codec == "rlev1" else _walk_rlev2)(s)
                dens = units * 1024 / max(int(out_b) // 32, 1)
        else:
            b = int(e.data[int(e.meta["comp_off"][0]) + 2])
            bt = (b >> 1) & 3
            share = bt * 0.5
            dens = (((b >> 3) & 31) + 257) / 286 if bt == 2 else 0.0
        want = [np.log2(1 + units), share, dens, 0.0]
        assert np.allclose(H[ti], want, rtol=1e-5, atol=1e-5), (it.codec, ti, H[ti], want)
    assert set(np.unique(T["codec"])) == {0, 1, 2, 3, 4}
