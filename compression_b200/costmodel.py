"""Learned task-cost model and the longest-predicted-first scheduler.

The model is the FP32 MLP 16 -> 64 -> 64 -> 1 of csrc/mlp.cu, trained on the
GPU by the library's own kernels (gd_mlp_train_step: forward, backward and
Adam in one launch per mini-batch) to predict log(decode time in ns) of a
batch task from its 16 header features (compression_b200.batch.task_features).
The training data are per-task times the batch decoder measures itself
(%globaltimer stamps around every task).

Scheduling: tasks are sorted by predicted cost, longest first, and fed to the
persistent decoder's work queue -- LPT list scheduling.  The static mapping
(task i -> warp i mod W) remains the fallback.
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
        torch = self.torch
        d_x = torch.from_numpy(self._norm(X)).to(self.dev)
        d_o = torch.empty(X.shape[0], dtype=torch.float32, device=self.dev)
        self.predict_device(d_x, X.shape[0], d_o)
        return d_o.cpu().numpy().astype(np.float64) + self.y_mu

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

def lpt_order(cost: np.ndarray):
    """Task order, longest predicted first (device int32 tensor)."""
    import torch
    return torch.from_numpy(np.argsort(-np.asarray(cost), kind="stable").astype(np.int32)).cuda()


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
    """[MLP inference -> longest-first sort -> persistent decode] captured in
    one CUDA graph over device-resident features; replay() decodes the batch."""

    def __init__(self, plan: B.Plan, model: CostModel, X: np.ndarray):
        import torch
        self.torch = torch
        self.plan = plan
        n = plan.tasks.size
        self.d_x = torch.from_numpy(model._norm(X)).cuda()
        self.d_pred = torch.empty(n, dtype=torch.float32, device="cuda")
        s = torch.cuda.Stream()
        # warm-up outside capture (first launches set kernel attributes)
        with torch.cuda.stream(s):
            model.predict_device(self.d_x, n, self.d_pred, s)
            order = torch.argsort(self.d_pred, descending=True).to(torch.int32)
            B.launch(plan, order, dynamic=True, timing=False, stream=s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            model.predict_device(self.d_x, n, self.d_pred, s)
            self.order = torch.argsort(self.d_pred, descending=True).to(torch.int32)
            B.launch(plan, self.order, dynamic=True, timing=False, stream=s)
        torch.cuda.synchronize()

    def replay(self) -> None:
        self.graph.replay()
