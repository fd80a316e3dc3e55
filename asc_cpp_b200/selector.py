"""Learned SpMV variant selector: data collection, training and installation.

The cost model is the library's own MLP (12 -> 64 -> 64 -> V, FP32), run by
its CUDA kernels (asc_sb_selector_forward / _backward / _adam): it predicts,
for each candidate variant, log(time) minus the matrix's mean log(time) over
the candidates, and the smallest prediction is the pick.  Training data comes
from the library's exhaustive autotuner (asc_sb_plan_autotune) run on seeded
synthetic matrices from four families -- banded, lognormal power-law,
block-diagonal with dense 8 x 8 blocks, uniform random -- with features from
the library's feature kernels (asc_sb_matrix_features).

Typical use::

    python -m asc_cpp_b200.selector collect --count 2000 --out timings.npz
    python -m asc_cpp_b200.selector train --data timings.npz --out weights.npz

and, in an application, ``install(context)`` to let plans created in
BACKEND_DEFAULT mode pick their variant with the shipped weights.
"""

from __future__ import annotations

import argparse
import ctypes
import os
import time

import numpy as np
import torch

from . import sparse_cuda as sc
from ._abi import Determinism, Variant

FEATURES = 12
HIDDEN = 64
# candidate variants, in output order: (variant, lanes)
VARIANTS: list[tuple[int, int]] = [(int(Variant.kWarpTiles), 0), (int(Variant.kMergePath), 0)] + \
    [(int(Variant.kVector), lanes) for lanes in (1, 2, 4, 8, 16, 32)] + \
    [(int(Variant.kRowSplit), 0)]
DEFAULT = 0  # the library's default variant (WARP_TILES) is output 0
FAMILIES = ("banded", "powerlaw", "blockdiag", "uniform")
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_weights.npz")


def param_count(v: int) -> int:
    return HIDDEN * FEATURES + HIDDEN + HIDDEN * HIDDEN + HIDDEN + v * HIDDEN + v


def _p(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


# ---- features ---------------------------------------------------------------

def matrix_features(context: sc.SparseCudaContext, matrix: sc.CudaCsrArray) -> torch.Tensor:
    """The twelve features of a device matrix (a device tensor)."""
    dev = torch.device("cuda", context.device)
    out = torch.empty(FEATURES, dtype=torch.float32, device=dev)
    scratch = torch.empty(8, dtype=torch.int64, device=dev)
    d = matrix.describe()
    context.check(context._lib.asc_sb_matrix_features(context.handle, ctypes.byref(d),
                                                      out.data_ptr(), scratch.data_ptr()))
    return out


# ---- the MLP on the library's kernels ----------------------------------------

class Mlp:
    """FP32 parameters on the GPU, trained with the library's kernels."""

    def __init__(self, context: sc.SparseCudaContext, n_outputs: int, seed: int = 0,
                 params: np.ndarray | None = None):
        self.context = context
        self.v = n_outputs
        dev = torch.device("cuda", context.device)
        if params is None:
            rng = np.random.default_rng(seed)
            parts = []
            for fan_out, fan_in in ((HIDDEN, FEATURES), (HIDDEN, HIDDEN), (n_outputs, HIDDEN)):
                parts.append(rng.standard_normal(fan_out * fan_in) * np.sqrt(2.0 / fan_in))
                parts.append(np.zeros(fan_out))
            params = np.concatenate(parts)
        assert params.size == param_count(n_outputs)
        self.params = torch.from_numpy(np.asarray(params, np.float32)).to(dev)

    def forward(self, x: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(y [batch, V], hidden [batch, 128]) for device features x [batch, 12]."""
        b = x.shape[0]
        hidden = torch.empty(b * 2 * HIDDEN, dtype=torch.float32, device=x.device)
        y = torch.empty(b, self.v, dtype=torch.float32, device=x.device)
        self.context.check(self.context._lib.asc_sb_selector_forward(
            self.context.handle, self.v, self.params.data_ptr(), x.data_ptr(), b,
            hidden.data_ptr(), y.data_ptr()))
        return y, hidden

    def gradient(self, x: torch.Tensor, target: torch.Tensor):
        """(gradient of the MSE loss, per-sample losses, y) for one batch."""
        b = x.shape[0]
        y, hidden = self.forward(x)
        grads = torch.empty_like(self.params)
        loss = torch.empty(b, dtype=torch.float32, device=x.device)
        scratch = torch.empty(b * (self.v + 2 * HIDDEN), dtype=torch.float32, device=x.device)
        self.context.check(self.context._lib.asc_sb_selector_backward(
            self.context.handle, self.v, self.params.data_ptr(), x.data_ptr(), b,
            hidden.data_ptr(), y.data_ptr(), target.data_ptr(), grads.data_ptr(),
            loss.data_ptr(), scratch.data_ptr()))
        return grads, loss, y

    def train(self, x: torch.Tensor, target: torch.Tensor, epochs: int = 3000,
              lr: float = 2e-3) -> list[float]:
        """Full-batch Adam; returns the mean loss every 100 epochs."""
        m = torch.zeros_like(self.params)
        s = torch.zeros_like(self.params)
        history = []
        for epoch in range(1, epochs + 1):
            grads, loss, _ = self.gradient(x, target)
            self.context.check(self.context._lib.asc_sb_selector_adam(
                self.context.handle, self.params.data_ptr(), grads.data_ptr(), m.data_ptr(),
                s.data_ptr(), self.params.numel(), ctypes.c_float(lr), ctypes.c_float(0.9),
                ctypes.c_float(0.999), ctypes.c_float(1e-8), epoch))
            if epoch % 100 == 0 or epoch == 1:
                history.append(float(loss.mean()))
        return history


def fold_normalisation(params: np.ndarray, mean: np.ndarray, std: np.ndarray,
                       v: int) -> np.ndarray:
    """Parameters that take raw features: W1' = W1 / std, b1' = b1 - W1' mean."""
    p = np.asarray(params, np.float64).copy()
    w1 = p[:HIDDEN * FEATURES].reshape(HIDDEN, FEATURES)
    b1 = p[HIDDEN * FEATURES:HIDDEN * FEATURES + HIDDEN]
    w1n = w1 / std[None, :]
    b1n = b1 - w1n @ mean
    p[:HIDDEN * FEATURES] = w1n.reshape(-1)
    p[HIDDEN * FEATURES:HIDDEN * FEATURES + HIDDEN] = b1n
    return p.astype(np.float32)


def targets(times: np.ndarray) -> np.ndarray:
    """log(time) minus the matrix's mean log(time) over the candidates."""
    lt = np.log(np.maximum(times, 1e-9))
    return (lt - lt.mean(axis=1, keepdims=True)).astype(np.float32)


def evaluate(picks: np.ndarray, times: np.ndarray) -> dict:
    """Slowdown of the picks against exhaustive autotuning, and their speedup
    over the default variant."""
    rows = np.arange(times.shape[0])
    t_pick = times[rows, picks]
    t_best = times.min(axis=1)
    t_default = times[:, DEFAULT]
    slow = t_pick / t_best
    return {
        "mean_slowdown_vs_exhaustive": float(slow.mean()),
        "geomean_slowdown_vs_exhaustive": float(np.exp(np.log(slow).mean())),
        "p90_slowdown_vs_exhaustive": float(np.quantile(slow, 0.9)),
        "exact_pick_fraction": float((picks == times.argmin(axis=1)).mean()),
        "geomean_speedup_vs_default": float(np.exp(np.log(t_default / t_pick).mean())),
        "total_time_speedup_vs_default": float(t_default.sum() / t_pick.sum()),
        "default_geomean_slowdown_vs_exhaustive": float(np.exp(np.log(t_default / t_best).mean())),
    }


def train_and_evaluate(context: sc.SparseCudaContext, data: dict, train_count: int = 1600,
                       epochs: int = 3000, seed: int = 0) -> tuple[np.ndarray, dict, list]:
    """Trains on the first train_count matrices, evaluates on the rest.
    Returns (parameters for raw features, held-out report, loss history)."""
    feats = np.asarray(data["features"], np.float64)
    times = np.asarray(data["times"], np.float64)
    v = times.shape[1]
    mean = feats[:train_count].mean(axis=0)
    std = feats[:train_count].std(axis=0)
    std[std < 1e-6] = 1.0
    dev = torch.device("cuda", context.device)
    xn = torch.from_numpy(((feats - mean) / std).astype(np.float32)).to(dev)
    t = torch.from_numpy(targets(times)).to(dev)
    mlp = Mlp(context, v, seed=seed)
    history = mlp.train(xn[:train_count].contiguous(), t[:train_count].contiguous(), epochs)
    raw = fold_normalisation(mlp.params.cpu().numpy(), mean, std, v)
    held = Mlp(context, v, params=raw)
    y, _ = held.forward(torch.from_numpy(feats[train_count:].astype(np.float32)).to(dev))
    picks = y.argmin(dim=1).cpu().numpy()
    report = evaluate(picks, times[train_count:])
    report["train_count"] = int(train_count)
    report["held_out_count"] = int(times.shape[0] - train_count)
    return raw, report, history


def install(context: sc.SparseCudaContext, path: str = WEIGHTS) -> None:
    """Installs trained weights on a context: plans created on it in
    BACKEND_DEFAULT mode with variant AUTO then pick their variant."""
    w = np.load(path)
    params = np.ascontiguousarray(w["params"], np.float32)
    variants = np.ascontiguousarray(w["variants"], np.int32)
    lanes = np.ascontiguousarray(w["lanes"], np.int32)
    context.check(context._lib.asc_sb_context_set_selector(
        context.handle, int(variants.size), params.ctypes.data, variants.ctypes.data,
        lanes.ctypes.data))


DEFAULT_INC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "host",
                           "selector_default.inc")


def export_c(path: str = WEIGHTS, out: str = DEFAULT_INC) -> str:
    """Writes the weights as the C++ tables the library installs on every new
    context (csrc/host/selector_default.inc)."""
    w = np.load(path)
    params = np.asarray(w["params"], np.float32)
    variants = np.asarray(w["variants"], np.int32)
    lanes = np.asarray(w["lanes"], np.int32)
    assert params.size == param_count(variants.size)
    lines = ["// Trained variant selector installed on every new context.  Generated by",
             "// `python -m asc_cpp_b200.selector export-c` from selector_weights.npz;",
             "// do not edit.",
             f"constexpr int kDefaultSelectorOutputs = {variants.size};",
             "constexpr int32_t kDefaultSelectorVariants[] = {" +
             ", ".join(str(int(v)) for v in variants) + "};",
             "constexpr int32_t kDefaultSelectorLanes[] = {" +
             ", ".join(str(int(v)) for v in lanes) + "};",
             "constexpr float kDefaultSelectorParams[] = {"]
    vals = [np.format_float_scientific(v, unique=True) + "f" if np.isfinite(v) else "0.0f"
            for v in params.astype(np.float32)]
    for i in range(0, len(vals), 6):
        lines.append("    " + ", ".join(vals[i:i + 6]) + ",")
    lines.append("};")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    return out


# ---- synthetic families (generated on the GPU) ----------------------------------

def _csr_from_keys(keys: torch.Tensor, n: int, dtype, gen) -> sc.CudaCsrArray:
    keys = torch.unique(keys)  # sorted, duplicates removed
    rows = keys // n
    cols = keys - rows * n
    counts = torch.bincount(rows, minlength=n)
    ptr = torch.zeros(n + 1, dtype=torch.int64, device=keys.device)
    torch.cumsum(counts, 0, out=ptr[1:])
    val = torch.randn(cols.numel(), generator=gen, device=keys.device,
                      dtype=torch.float64).to(dtype)
    return sc.CudaCsrArray(n, n, ptr, cols.contiguous(), val)


def family_matrix(family: str, n: int, rng: np.random.Generator, dtype, nnz_cap: int,
                  device) -> sc.CudaCsrArray:
    """One seeded synthetic matrix of a family, n x n, about nnz_cap entries
    at most."""
    gen = torch.Generator(device=device)
    gen.manual_seed(int(rng.integers(1 << 62)))
    if family == "banded":
        hb = int(rng.integers(1, 65))
        hb = max(1, min(hb, nnz_cap // (2 * n) - 1))
        r = torch.arange(n, device=device)
        offs = torch.arange(-hb, hb + 1, device=device)
        c = r[:, None] + offs[None, :]
        ok = (c >= 0) & (c < n)
        rr = r[:, None].expand_as(c)[ok]
        keys = rr * n + c[ok]
        n_fill = int(round(0.01 * keys.numel()))
        fr = torch.randint(0, n, (n_fill,), generator=gen, device=device)
        fc = torch.randint(0, n, (n_fill,), generator=gen, device=device)
        keys = torch.cat([keys, fr * n + fc])
        return _csr_from_keys(keys, n, dtype, gen)
    if family == "powerlaw":
        mean = float(rng.uniform(2.0, 64.0))
        mean = min(mean, nnz_cap / n)
        sigma = float(rng.uniform(0.5, 2.0))
        mu = np.log(mean) - sigma * sigma / 2
        lengths = torch.exp(mu + sigma * torch.randn(n, generator=gen, device=device,
                                                     dtype=torch.float64))
        lengths = torch.clamp(torch.round(lengths), 1, min(65536, n)).long()
        rows = torch.repeat_interleave(torch.arange(n, device=device), lengths)
        cols = torch.randint(0, n, (rows.numel(),), generator=gen, device=device)
        return _csr_from_keys(rows * n + cols, n, dtype, gen)
    if family == "blockdiag":
        n = max(8, n // 8 * 8)
        nb = n // 8
        k = int(rng.integers(1, 5))
        k = max(1, min(k, nnz_cap // (8 * n)))
        brow = torch.arange(nb, device=device).repeat_interleave(k)
        bcol = torch.randint(0, nb, (nb * k,), generator=gen, device=device)
        bcol.view(nb, k)[:, 0] = torch.arange(nb, device=device)  # the diagonal block
        i = torch.arange(8, device=device)
        rr = (brow[:, None, None] * 8 + i[None, :, None]).expand(-1, 8, 8)
        cc = (bcol[:, None, None] * 8 + i[None, None, :]).expand(-1, 8, 8)
        return _csr_from_keys((rr * n + cc).reshape(-1), n, dtype, gen)
    if family == "uniform":
        density = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-2))))
        lam = min(density * n, nnz_cap / n)
        lengths = torch.poisson(torch.full((n,), lam, device=device, dtype=torch.float64),
                                generator=gen).long()
        lengths = torch.clamp(lengths, 0, n)
        rows = torch.repeat_interleave(torch.arange(n, device=device), lengths)
        cols = torch.randint(0, n, (rows.numel(),), generator=gen, device=device)
        return _csr_from_keys(rows * n + cols, n, dtype, gen)
    raise ValueError(family)


def collect(count: int = 2000, seed: int = 4, min_rows: int = 10_000,
            max_rows: int = 10_000_000, nnz_cap: int = 20_000_000, reps_floor: int = 5,
            log_every: int = 100) -> dict:
    """Features and exhaustive-autotune times (ms, y = A x) of `count` seeded
    matrices: families in turn, rows log-uniform in [min_rows, max_rows],
    FP32 or FP64 at random, nnz limited to about nnz_cap."""
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(seed)
    ctx = sc.SparseCudaContext.Create(0, stream=torch.cuda.default_stream(0),
                                      determinism=Determinism.kBackendDefault)
    variants = np.array([v for v, _ in VARIANTS], np.int32)
    lanes = np.array([l for _, l in VARIANTS], np.int32)
    feats = np.zeros((count, FEATURES), np.float32)
    times = np.zeros((count, len(VARIANTS)), np.float32)
    meta = np.zeros((count, 4), np.int64)  # family, rows, nnz, element bytes
    t0 = time.time()
    for i in range(count):
        family = FAMILIES[i % len(FAMILIES)]
        n = int(np.exp(rng.uniform(np.log(min_rows), np.log(max_rows))))
        dtype = torch.float64 if rng.random() < 0.5 else torch.float32
        m = family_matrix(family, n, rng, dtype, nnz_cap, dev)
        feats[i] = matrix_features(ctx, m).cpu().numpy()
        x = (torch.rand(m.columns, generator=None, device=dev, dtype=torch.float64) * 2 - 1).to(dtype)
        y = torch.zeros(m.rows, dtype=dtype, device=dev)
        plan = sc.CsrPlan(ctx, m)
        reps = max(reps_floor, int(2_000_000 // max(m.nnz, 1)))
        reps = min(reps, 200)
        ms = np.zeros(len(VARIANTS), np.float32)
        xv = sc.CudaStridedVectorView(x, m.columns, writable=False)
        yv = sc.CudaStridedVectorView(y, m.rows)
        xd, yd = xv.describe(), yv.describe()
        xd.writable = 0
        ctx.check(ctx._lib.asc_sb_plan_autotune(ctx.handle, plan.handle, ctypes.byref(xd),
                                                ctypes.byref(yd), len(VARIANTS),
                                                variants.ctypes.data, lanes.ctypes.data, reps,
                                                ms.ctypes.data))
        times[i] = ms
        meta[i] = (FAMILIES.index(family), m.rows, m.nnz, 8 if dtype == torch.float64 else 4)
        plan.close()
        del m, x, y
        if log_every and (i + 1) % log_every == 0:
            print(f"# collected {i + 1}/{count} in {time.time() - t0:.0f}s", flush=True)
    ctx.close()
    return {"features": feats, "times": times, "meta": meta,
            "variants": variants, "lanes": lanes, "nnz_cap": np.array([nnz_cap]),
            "seed": np.array([seed])}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=2000)
    c.add_argument("--seed", type=int, default=4)
    c.add_argument("--nnz-cap", type=int, default=20_000_000)
    c.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--out", required=True)
    t.add_argument("--train-count", type=int, default=1600)
    t.add_argument("--epochs", type=int, default=3000)
    e = sub.add_parser("export-c")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--out", default=DEFAULT_INC)
    a = ap.parse_args()
    if a.cmd == "export-c":
        print(export_c(a.weights, a.out))
        return
    if a.cmd == "collect":
        np.savez_compressed(a.out, **collect(a.count, a.seed, nnz_cap=a.nnz_cap))
        return
    data = dict(np.load(a.data))
    ctx = sc.SparseCudaContext.Create(0, stream=torch.cuda.default_stream(0))
    raw, report, history = train_and_evaluate(ctx, data, a.train_count, a.epochs)
    np.savez(a.out, params=raw, variants=data["variants"], lanes=data["lanes"])
    print({"loss_history": history[::5], **report})


if __name__ == "__main__":
    main()
