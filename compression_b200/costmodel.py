"""Learned task-cost model and the longest-predicted-first scheduler.

The model is the FP32 MLP 16 -> 64 -> 64 -> 1 of csrc/mlp.cu, trained on the
GPU by the library's own kernels (gd_mlp_train_step: forward, backward and
Adam in one launch per mini-batch) to predict log(decode time in ns) of a
batch task from its 16 header features (compression_b200.batch.task_features).
The training data are per-task times the batch decoder measures itself
(%globaltimer stamps around every task).

Scheduling: tasks are sorted by predicted cost, longest first, and fed to the
persistent decoder's work queue -- LPT list scheduling.  The lane tasks of one
RLE chunk (the 32 tasks that read the same interleaved block) are ordered as
one group, keyed by their largest prediction, so that they stay adjacent in
the queue and run side by side: each of them reads 4 bytes of every 128-byte
row of the block, and when they run apart every one of them fetches the rows
again (ordering every task by its own measured time was slower than ordering
by output bytes for that reason).  Inside bands of a factor of 2 of
predicted time the order runs one codec after another, so that an SM's warps
mostly run one decoder's code: the batch kernel holds all five decoders,
more code than the instruction cache keeps.  The static mapping (task i ->
warp i mod W) remains the fallback.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import batch as B
from . import codecs as cc
from ._lib import lib

N_IN = 16


class CostModel:
    def __init__(self, seed: int = 0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.np_ = int(lib().gd_mlp_num_params())
        rng = np.random.default_rng(seed)
        p = np.zeros(self.np_, np.float32)
        # He-uniform init, zero biases
        o = 0
        for fan_in, fan_out in ((N_IN, 64), (64, 64), (64, 1)):
            lim = np.sqrt(6.0 / fan_in)
            p[o:o + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out)
            o += fan_in * fan_out + fan_out
        self.params = torch.from_numpy(p).to(self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.mu = np.zeros(N_IN, np.float32)
        self.sd = np.ones(N_IN, np.float32)
        self.y_mu = 0.0

    # ---- feature normalisation ----
    def _norm(self, X: np.ndarray) -> np.ndarray:
        return ((X - self.mu) / self.sd).astype(np.float32)

    def fit_normaliser(self, X: np.ndarray, y: np.ndarray) -> None:
        self.mu = X.mean(0).astype(np.float32)
        sd = X.std(0).astype(np.float32)
        sd[sd < 1e-6] = 1.0
        self.sd = sd
        self.mu[-1] = 0.0  # keep the constant feature at 1
        self.sd[-1] = 1.0
        self.y_mu = float(y.mean())

    # ---- kernels ----
    def predict_device(self, d_x, n: int, d_out, stream=None) -> None:
        """Raw network output for normalised device features (for graph capture)."""
        s = stream.cuda_stream if stream is not None else self.torch.cuda.current_stream().cuda_stream
        cc.check(lib().gd_mlp_predict(C.c_void_p(self.params.data_ptr()), C.c_void_p(d_x.data_ptr()), n,
                                      C.c_void_p(d_out.data_ptr()), C.c_void_p(s)), "gd_mlp_predict")

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Predicted log(ns) per row of raw features X."""
        return self.predict32(X).astype(np.float64)

    def predict32(self, X: np.ndarray) -> np.ndarray:
        """Predicted log(ns) in float32, computed as the scheduling graph does
        (network output + mean target, in float32)."""
        torch = self.torch
        d_x = torch.from_numpy(self._norm(X)).to(self.dev)
        d_o = torch.empty(X.shape[0], dtype=torch.float32, device=self.dev)
        self.predict_device(d_x, X.shape[0], d_o)
        return (d_o + np.float32(self.y_mu)).cpu().numpy()

    def grad(self, d_x, d_y, d_idx, nb: int):
        """Gradient of the mini-batch MSE (normalised targets), on the device."""
        torch = self.torch
        g = torch.empty(self.np_, dtype=torch.float32, device=self.dev)
        loss = torch.empty(1, dtype=torch.float32, device=self.dev)
        s = torch.cuda.current_stream().cuda_stream
        cc.check(lib().gd_mlp_train_step(C.c_void_p(self.params.data_ptr()), None, None, C.c_void_p(d_x.data_ptr()),
                                         C.c_void_p(d_y.data_ptr()), C.c_void_p(d_idx.data_ptr()), nb, 0.0, 0.9,
                                         0.999, 1e-8, 0, C.c_void_p(g.data_ptr()), C.c_void_p(loss.data_ptr()),
                                         C.c_void_p(s)), "gd_mlp_train_step")
        return g, loss

    def train(self, X: np.ndarray, y: np.ndarray, epochs: int = 20, batch: int = 256, lr: float = 2e-3,
              seed: int = 0, weights: np.ndarray | None = None) -> list[float]:
        """Adam on log-time targets; returns the mean loss of every epoch.
        weights (optional, one per row): every epoch draws its n rows with
        replacement in proportion to them (so the squared error of a row
        counts in proportion to its weight); without them each row is seen
        once per epoch."""
        torch = self.torch
        if self.step == 0:
            self.fit_normaliser(X, y)
        d_x = torch.from_numpy(self._norm(X)).to(self.dev)
        d_y = torch.from_numpy((y - self.y_mu).astype(np.float32)).to(self.dev)
        n = X.shape[0]
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        losses = []
        L = lib()
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        d_loss = torch.zeros(max(1, (n + batch - 1) // batch), dtype=torch.float32, device=self.dev)
        d_w = None
        if weights is not None:
            d_w = torch.from_numpy(np.asarray(weights, np.float64) / np.sum(weights)).to(self.dev)
        for _ in range(epochs):
            if d_w is None:
                perm = torch.randperm(n, generator=gen, device=self.dev).to(torch.int32)
            else:
                perm = torch.multinomial(d_w, n, replacement=True, generator=gen).to(torch.int32)
            nsteps = (n + batch - 1) // batch
            for k in range(nsteps):
                nb = min(batch, n - k * batch)
                self.step += 1
                idx = perm[k * batch:k * batch + nb]
                cc.check(L.gd_mlp_train_step(C.c_void_p(self.params.data_ptr()), C.c_void_p(self.m.data_ptr()),
                                             C.c_void_p(self.v.data_ptr()), C.c_void_p(d_x.data_ptr()),
                                             C.c_void_p(d_y.data_ptr()), C.c_void_p(idx.data_ptr()), nb, lr, 0.9,
                                             0.999, 1e-8, self.step, None,
                                             C.c_void_p(d_loss.data_ptr() + 4 * k), s), "train")
            losses.append(float(d_loss[:nsteps].mean().item()))
        return losses

    # ---- persistence ----
    def to_json(self) -> str:
        return json.dumps({"params": self.params.cpu().numpy().tolist(), "mu": self.mu.tolist(),
                           "sd": self.sd.tolist(), "y_mu": self.y_mu})

    def load_json(self, s: str) -> None:
        d = json.loads(s)
        self.params = self.torch.tensor(d["params"], dtype=self.torch.float32, device=self.dev)
        self.mu = np.array(d["mu"], np.float32)
        self.sd = np.array(d["sd"], np.float32)
        self.y_mu = float(d["y_mu"])


# --------------------------------------------------------------------------
# scheduling
# --------------------------------------------------------------------------

def task_groups(plan: B.Plan) -> np.ndarray:
    """Group id of every task: a run of consecutive tasks that read the same
    source block (the lane tasks of one RLE chunk, which the plan lists
    together) is one group; every other task is a group alone.  Ids count up
    in task order, so a group's tasks are contiguous."""
    src = plan.tasks["src"]
    new = np.ones(src.size, bool)
    new[1:] = src[1:] != src[:-1]
    return (np.cumsum(new) - 1).astype(np.int64)


def group_max(cost: np.ndarray, groups: np.ndarray) -> np.ndarray:
    """Every task's cost replaced by the largest cost in its group."""
    cost = np.asarray(cost, np.float64)
    k = np.full(int(groups.max()) + 1 if groups.size else 0, -np.inf)
    np.maximum.at(k, groups, cost)
    return k[groups]


BAND = float(np.log(2.0))  # width of a cost band (natural-log units): a factor of 2


def band_sort_key(cost: np.ndarray, codec: np.ndarray, band: float = BAND) -> np.ndarray:
    """Ascending int32 sort key of the banded longest-first order of log
    costs (float32): bands of `band` (a cost factor of e^band), the costliest
    band first; inside a band one codec after another; inside that, the
    costliest first (the cost's place in its band in 21 bits).  Runs of one
    codec keep the warps of an SM on one decoder's code (the batch kernel
    holds all five, more than the instruction cache)."""
    c = np.asarray(cost, np.float32)
    t = c / np.float32(band)
    fl = np.floor(t)
    k1 = 127 - np.clip(fl, 0, 127).astype(np.int32)
    q = np.clip(np.floor((np.float32(1.0) - (t - fl)) * np.float32(1 << 21)), 0, (1 << 21) - 1).astype(np.int32)
    return (k1 << 24) | (np.asarray(codec, np.int32) << 21) | q


def lpt_order_host(cost: np.ndarray, groups: np.ndarray | None = None, codec: np.ndarray | None = None,
                   band: float = BAND) -> np.ndarray:
    """Task order, longest predicted first; with groups, a group's tasks share
    its largest cost and stay together, in task order (ties keep task order);
    with codec (and log costs), the banded order of band_sort_key."""
    if codec is not None:
        c = np.asarray(cost, np.float32)
        if groups is not None:
            c = group_max(c, groups).astype(np.float32)
        return np.argsort(band_sort_key(c, codec, band), kind="stable").astype(np.int32)
    key = np.asarray(cost, np.float64) if groups is None else group_max(cost, groups)
    return np.argsort(-key, kind="stable").astype(np.int32)


def lpt_order(cost: np.ndarray, groups: np.ndarray | None = None, codec: np.ndarray | None = None,
              band: float = BAND):
    """lpt_order_host as a device int32 tensor (the batch decoder's order)."""
    import torch
    return torch.from_numpy(lpt_order_host(cost, groups, codec, band)).cuda()


def measure_tasks(plan: B.Plan, seed: int = 0, reps: int = 1) -> np.ndarray:
    """Per-task decode times (ns) measured by the batch decoder itself, in a
    random task order through the work queue (median over reps)."""
    import torch
    n = plan.tasks.size
    rng = np.random.default_rng(seed)
    ds = []
    for r in range(reps):
        order = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda()
        B.launch(plan, order, dynamic=True, timing=True)
        torch.cuda.synchronize()
        ds.append(B.task_durations_ns(plan))
    return np.median(np.stack(ds), axis=0)


class GraphSchedule:
    """[MLP inference -> group maximum -> longest-first sort -> persistent
    decode] captured in one CUDA graph over device-resident features;
    replay() decodes the batch.  groups: task_groups(plan) (default; groups
    must be contiguous runs of tasks), or None to order every task by its own
    prediction; banded: the order of band_sort_key (codec runs inside cost
    bands of a factor of 2), else plain longest first."""

    _AUTO = object()

    def __init__(self, plan: B.Plan, model: CostModel, X: np.ndarray, groups=_AUTO, banded: bool = True,
                 band: float = BAND):
        import torch
        self.torch = torch
        self.plan = plan
        n = plan.tasks.size
        if groups is GraphSchedule._AUTO:
            groups = task_groups(plan)
        self.d_x = torch.from_numpy(model._norm(X)).cuda()
        # the group maximum as a padded gather (no atomics, no host syncs, so
        # it can be captured): row g of d_gidx lists group g's tasks, padded
        # with n, which points at a -inf after the predictions
        self.d_pred = torch.full((n + 1,), float("-inf"), dtype=torch.float32, device="cuda")
        self.d_grp = self.d_gidx = None
        if groups is not None:
            groups = np.asarray(groups, np.int64)
            ng = int(groups.max()) + 1 if n else 0
            cnt = np.bincount(groups, minlength=ng)
            first = np.concatenate([[0], np.cumsum(cnt)[:-1]])
            order = np.argsort(groups, kind="stable")  # tasks grouped, in task order
            gidx = np.full((ng, int(cnt.max()) if ng else 1), n, np.int64)
            gidx[groups[order], np.arange(n) - first[groups[order]]] = order
            self.d_grp = torch.from_numpy(groups).cuda()
            self.d_gidx = torch.from_numpy(gidx).cuda()

        self.d_codec = (torch.from_numpy(plan.tasks["codec"].astype(np.int32) << 21).cuda() if banded else None)
        y_mu = float(np.float32(model.y_mu))

        def order_of():
            key = self.d_pred[:n]
            if self.d_grp is not None:
                key = self.d_pred[self.d_gidx].amax(dim=1)[self.d_grp]
            if self.d_codec is None:
                return torch.argsort(key, descending=True, stable=True).to(torch.int32)
            # band_sort_key on the device (the same float32 operations)
            t = (key + y_mu) / band
            fl = torch.floor(t)
            k1 = 127 - fl.clamp(0, 127).to(torch.int32)
            q = torch.floor((1.0 - (t - fl)) * float(1 << 21)).clamp(0, (1 << 21) - 1).to(torch.int32)
            skey = (k1 << 24) | self.d_codec | q
            return torch.argsort(skey, stable=True).to(torch.int32)

        s = torch.cuda.Stream()
        # warm-up outside capture (first launches set kernel attributes)
        with torch.cuda.stream(s):
            model.predict_device(self.d_x, n, self.d_pred, s)
            B.launch(plan, order_of(), dynamic=True, timing=False, stream=s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            model.predict_device(self.d_x, n, self.d_pred, s)
            self.order = order_of()
            B.launch(plan, self.order, dynamic=True, timing=False, stream=s)
        torch.cuda.synchronize()

    def replay(self) -> None:
        self.graph.replay()
