"""The autotuner on the device: every candidate of every knob decodes
bit-identically (the tuner checks that itself), the chosen value is one of
the candidates, decoding with it still matches the oracle, and remembered
choices are re-applied from the cache file."""
import numpy as np
import pytest

import compression_b200.autotune as at
import compression_b200.batch as B
import compression_b200.codecs as cc
import oracle

pytestmark = pytest.mark.gpu


def _cases():
    raw_d = cc.gen_markov_copy(3, 3 << 20, 32768)
    sizes = cc.loguniform_sizes(4, 40, 4096, 256 << 10, raw_d.size)
    oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    return [
        (cc.brle_encode(cc.gen_brle_bytes(1, 4 << 20)), None),
        (cc.rlev1_encode(cc.gen_rlev1_ints(2, 1 << 20), 128 * 1024, 128, 4), None),
        (cc.rlev2_encode(cc.gen_rlev2_ints(3, 1 << 19), 256 * 1024, 32), None),
        (cc.lzss_encode(cc.gen_markov_copy(5, 2 << 20, 4096), 64 * 1024), None),
        (cc.deflate_encode(raw_d, oo), None),
    ]


def test_tune_every_codec(cuda, tmp_path):
    import torch
    tuner = at.Tuner(tmp_path / "tune.json", cuda)
    saved = {k: at.get_knob(k) for k, _ in at.KNOBS.values()}
    try:
        for enc, _ in _cases():
            job = cc.DeviceJob(enc, cuda)
            res = tuner.tune_job(job, reps=2)
            knob, values = at.KNOBS[enc.codec]
            assert res["value"] in values and at.get_knob(knob) == res["value"]
            job.d_out.zero_()
            job.launch()
            torch.cuda.synchronize()
            rc, ref = oracle.decode(enc)
            assert rc == 0 and (job.status() == 0).all() and np.array_equal(job.output(), ref)
        tuner.save()
        # a fresh tuner applies the remembered choices
        for k in saved:
            at.set_knob(k, 0)
        t2 = at.Tuner(tmp_path / "tune.json", cuda)
        enc = _cases()[0][0]
        assert t2.apply("brle", enc.n_out)
        assert at.get_knob(at.TUNE_BRLE_BLOCKS_PER_SM) == tuner.results[tuner.key("brle", enc.n_out)]["value"]
    finally:
        for k, v in saved.items():
            at.set_knob(k, v)


def test_tune_batch_blocks_per_sm(cuda):
    items = B.make_mixed_batch(21, 60, 12 << 20)
    plan = B.build_plan(items, cuda)
    res = at.Tuner(None, cuda).tune_batch(plan, candidates=[1, 2, 0], reps=2)
    assert res["blocks_per_sm"] in (0, 1, 2)
    plan.d_out.zero_()
    B.launch(plan, None, dynamic=True, timing=False, blocks_per_sm=res["blocks_per_sm"])
    import torch
    torch.cuda.synchronize()
    assert B.verify(plan)
