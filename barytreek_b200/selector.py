"""Learned interpolation-degree selector: data generation, training, weights.

The network (16 -> 64 -> 64 -> 9, ReLU, BF16 weights, FP32 accumulation) runs
in the library's own CUDA kernels for inference, forward, backward and Adam
(btk_mlp_*); this module drives them. Training data are error samples the
treecode generates itself (btk_plan_error_samples): for sampled far-field
pairs of a BTK_DEGREE_PER_PAIR plan, the relative error of the pair's
contribution at K target points at every degree, against the FP64 direct sum
over the source panel's points.

Weight files are versioned .npz archives: params (FP32, 5833), norm (34),
version, and provenance (families, samples, validation loss).
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import _lib
from ._lib import check, load, ptr

N_FEATURES, N_HIDDEN, N_OUT, DEG_LO = 16, 64, 9, 4
WEIGHTS_VERSION = 1
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_weights.npz")
# The reference's 3-D "velocity" kernel q (t-s)/(r^2+eps^2) has its own far-field
# error behaviour; its network is trained on its own samples.
VEL_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_weights_vel.npz")


def weights_for(kind: int) -> str:
    """The weight file for a kernel kind (VEL has its own; POT and FIELD share one)."""
    return VEL_WEIGHTS if kind == _lib.KIND_VEL else DEFAULT_WEIGHTS


def param_count() -> int:
    return int(load().btk_selector_param_count())


def init_params(rng: np.random.Generator) -> np.ndarray:
    """He-initialised FP32 parameters in the library's layout."""
    p = []
    for fan_out, fan_in in ((N_HIDDEN, N_FEATURES), (N_HIDDEN, N_HIDDEN), (N_OUT, N_HIDDEN)):
        p.append((rng.standard_normal((fan_out, fan_in)) * np.sqrt(2.0 / fan_in)).ravel())
        p.append(np.zeros(fan_out))
    out = np.concatenate(p).astype(np.float32)
    assert out.size == param_count()
    return out


class Selector:
    """Parameters + normalisation; creates the device selector on demand."""

    def __init__(self, params: np.ndarray, norm: np.ndarray, meta: dict | None = None):
        self.params = np.ascontiguousarray(params, np.float32)
        self.norm = np.ascontiguousarray(norm, np.float32)
        self.meta = meta or {}
        self._h = ctypes.c_void_p()

    @classmethod
    def load(cls, path: str | None = None, kind: int = _lib.KIND_FIELD) -> "Selector":
        """Loads a weight file (default: the one for ``kind``)."""
        path = path or weights_for(kind)
        z = np.load(path, allow_pickle=False)
        if int(z["version"]) != WEIGHTS_VERSION:
            raise ValueError(f"{path}: weight file version {int(z['version'])}, expected {WEIGHTS_VERSION}")
        meta = {k: z[k].item() if z[k].ndim == 0 else z[k] for k in z.files if k not in ("params", "norm")}
        return cls(z["params"], z["norm"], meta)

    def save(self, path: str) -> None:
        extra = {k: np.asarray(v) for k, v in self.meta.items() if k != "version"}
        np.savez(path, params=self.params, norm=self.norm, version=np.asarray(WEIGHTS_VERSION), **extra)

    def handle(self):
        if not self._h:
            check(load().btk_selector_create(ctypes.byref(self._h), ptr(self.params), ptr(self.norm)))
        return self._h

    def __del__(self):
        try:
            if self._h:
                load().btk_selector_destroy(self._h)
        except Exception:
            pass


# ------------------------------------------------------------------ sampling
def _subtree_leaves(panels, root):
    out, stack = [], [root]
    while stack:
        p = stack.pop()
        if panels["is_leaf"][p]:
            out.append(p)
        else:
            stack.extend(int(c) for c in panels["child"][p])
    return out


def generate_samples(tc, charges, n_samples: int, K: int = 32, seed: int = 0, batch: int = 4096):
    """Features and log10 errors (degrees degree_min..interp_degree) of
    n_samples random far-field pairs of a per-pair Treecode."""
    import torch
    L = load()
    rng = np.random.default_rng(seed)
    if tc.stats()["leaf_far_pairs"]:
        raise ValueError("error samples index the PC, CP and CC lists: use a plan without leaf_far_pairs")
    n_pairs = ctypes.c_int()
    check(L.btk_plan_pair_count(tc._plan, ctypes.byref(n_pairs)))
    n_pairs = n_pairs.value
    if n_pairs == 0:
        return np.zeros((0, N_FEATURES), np.float32), np.zeros((0, 0), np.float32)
    q = torch.as_tensor(np.ascontiguousarray(charges, np.float64), device=tc.device)
    s = tc._s
    zs = ptr(s[2]) if tc.dim == 3 else None
    zt = ptr(tc._t[2]) if tc.dim == 3 else None
    feat = torch.empty((n_pairs, N_FEATURES), dtype=torch.float32, device=tc.device)
    stream = torch.cuda.current_stream(tc.device).cuda_stream
    check(L.btk_plan_pair_features(tc._plan, ptr(s[0]), ptr(s[1]), zs, ptr(q), ptr(feat), stream))
    feat = feat.cpu().numpy()
    # The total solution at the plan degree (every pair at the highest degree):
    # pair errors are measured relative to it, which is what the global
    # tolerance constrains.
    ref = tc.solve(q)
    # pair table (PC, CP, CC) -> (target, source panels)
    pp, pc, cp, cc = tc.lists
    tg = np.concatenate([pc["target_panel"], cp["target_panel"], cc["target_panel"]])
    sr = np.concatenate([pc["source_panel"], cp["source_panel"], cc["source_panel"]])
    tt, st = tc.tree_t, (tc.tree_s or tc.tree_t)
    # empty leaves appear in the lists; their pairs carry no signal
    valid = np.flatnonzero((tt.panels["point_count"][tg] > 0) & (st.panels["point_count"][sr] > 0))
    if len(valid) == 0:
        return np.zeros((0, N_FEATURES), np.float32), np.zeros((0, 0), np.float32)
    pick = valid[rng.choice(len(valid), size=min(n_samples, len(valid)), replace=False)]
    n_deg = tc.cfg.interp_degree - tc.degree_min + 1
    errs = np.zeros((len(pick), n_deg), np.float32)
    leaves_cache_t, leaves_cache_s = {}, {}
    for b0 in range(0, len(pick), batch):
        idx = pick[b0:b0 + batch]
        tgt_orig = np.zeros((len(idx), K), np.int32)
        csr, leaves = [0], []
        for j, p in enumerate(idx):
            T = int(tg[p])
            if T not in leaves_cache_t:
                lv = _subtree_leaves(tt.panels, T)
                pts = np.concatenate([tt.panel_points_inside[l, :tt.panels["point_count"][l]] for l in lv])
                leaves_cache_t[T] = pts
            pts = leaves_cache_t[T]
            tgt_orig[j] = pts[rng.integers(0, len(pts), K)]
            S = int(sr[p])
            if S not in leaves_cache_s:
                leaves_cache_s[S] = np.asarray(_subtree_leaves(st.panels, S), np.int32)
            leaves.append(leaves_cache_s[S])
            csr.append(csr[-1] + len(leaves_cache_s[S]))
        csr = np.asarray(csr, np.int32)
        leaves = np.concatenate(leaves).astype(np.int32)
        out = np.zeros((len(idx), n_deg), np.float32)
        pi = np.ascontiguousarray(idx, np.int32)
        check(L.btk_plan_error_samples(tc._plan, ptr(tc._t[0]), ptr(tc._t[1]), zt, ptr(s[0]), ptr(s[1]), zs, ptr(q),
                                       len(idx), ptr(pi), K, ptr(tgt_orig), ptr(csr), ptr(leaves), ptr(ref), ptr(out),
                                       stream))
        errs[b0:b0 + len(idx)] = out
    return feat[pick], errs


def to_targets(errs: np.ndarray, degree_min: int, degree_max: int):
    """Map errors at degrees degree_min..degree_max onto the network's 9
    outputs (degrees 4..12) with a mask for degrees that were not sampled.
    Errors are clamped to [-16, 1] (log10)."""
    n = len(errs)
    y = np.zeros((n, N_OUT), np.float32)
    m = np.zeros((n, N_OUT), np.float32)
    for d in range(max(DEG_LO, degree_min), min(DEG_LO + N_OUT - 1, degree_max) + 1):
        y[:, d - DEG_LO] = np.clip(errs[:, d - degree_min], -16.0, 1.0)
        m[:, d - DEG_LO] = 1.0
    return y, m


# ------------------------------------------------------------------ training
def train(X, Y, M, *, epochs=40, batch=4096, lr=2e-3, seed=0, val_frac=0.1, device="cuda", log=None):
    """Trains on the GPU with btk_mlp_gradient / btk_mlp_adam. Returns a Selector."""
    import torch
    L = load()
    rng = np.random.default_rng(seed)
    n = len(X)
    perm = rng.permutation(n)
    n_val = max(1, int(n * val_frac))
    vi, ti = perm[:n_val], perm[n_val:]
    xm, xs = X[ti].mean(0), X[ti].std(0) + 1e-6
    w = M[ti] > 0
    ym = float(Y[ti][w].mean())
    ys = float(Y[ti][w].std() + 1e-6)
    norm = np.concatenate([xm, xs, [ym, ys]]).astype(np.float32)
    Xn = ((X - xm) / xs).astype(np.float32)
    Yn = ((Y - ym) / ys * (M > 0)).astype(np.float32)
    dev = torch.device(device)
    tX, tY, tM = (torch.from_numpy(a).to(dev) for a in (Xn, Yn, M.astype(np.float32)))
    P = param_count()
    master = torch.from_numpy(init_params(rng)).to(dev)
    wbf = torch.empty(P, dtype=torch.bfloat16, device=dev)
    wbf.copy_(master.to(torch.bfloat16))
    mom, vel, grad = (torch.zeros(P, dtype=torch.float32, device=dev) for _ in range(3))
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    work = torch.empty(batch * (4 * N_HIDDEN + N_OUT), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    step = 0
    ti_t = torch.from_numpy(ti).to(dev)
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        order = ti_t[torch.randperm(len(ti), device=dev)]
        tot, nb = 0.0, 0
        for b0 in range(0, len(ti) - batch + 1, batch):
            sel = order[b0:b0 + batch]
            xb, yb, mb = tX[sel].contiguous(), tY[sel].contiguous(), tM[sel].contiguous()
            check(L.btk_mlp_gradient(ptr(wbf), batch, ptr(xb), ptr(yb), ptr(mb), ptr(grad), ptr(loss), ptr(work),
                                     stream))
            step += 1
            lr_t = lr * 0.5 * (1 + np.cos(np.pi * min(1.0, ep / max(1, epochs))))
            check(L.btk_mlp_adam(ptr(master), ptr(wbf), ptr(grad), ptr(mom), ptr(vel), step, ctypes.c_float(lr_t),
                                 stream))
            tot += float(loss.item()) if (b0 // batch) % 16 == 0 else 0.0
            nb += 1 if (b0 // batch) % 16 == 0 else 0
        val = validation_loss(wbf, tX[vi], tY[vi], tM[vi], ys)
        hist.append((ep, tot / max(nb, 1), val))
        if log:
            log(f"epoch {ep:3d} train {tot / max(nb, 1):.4f} val rmse(log10) {val:.4f} ({time.time() - t0:.1f}s)")
    params = master.cpu().numpy().astype(np.float32)
    meta = {"samples": n, "val_rmse_log10": hist[-1][2] if hist else float("nan"), "epochs": epochs}
    return Selector(params, norm, meta)


def validation_loss(wbf, xv, yv, mv, ys):
    """RMSE of the predicted log10 errors on the masked validation targets."""
    import torch
    out = torch.empty_like(yv)
    check(load().btk_mlp_forward(ptr(wbf), len(xv), ptr(xv.contiguous()), ptr(out), None))
    torch.cuda.synchronize()
    d = (out - yv) * mv
    return float(torch.sqrt((d * d).sum() / mv.sum()).item() * ys)
