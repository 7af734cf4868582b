"""Learned surrogate of per-SDS log-reflectance, with plain MC as fallback.

Pipeline (all GPU work through the library's C ABI):
  1. labels: a set of baseline tissues is walked and replayed
     (Simulation.run / replay); White-MC relabelling (wmc.rescale) turns
     each replay into the reflectance of many (mua, mus) combinations
     around it -- mua anywhere in its range (an exact, well-conditioned
     reweighting), mus within a few percent of the baseline (its
     reweighting grows with the interaction count);
  2. training: an ensemble of MLPs (25 features = 5 layers x height, mua,
     mus, n, g -> log-reflectance per SDS) trained by the library's BF16
     tensor-core forward/backward kernels with Adam (MLP class);
  3. serving: queries inside the training hull whose ensemble members
     agree are answered by the network; the others fall back to plain MC
     (the batched walk) at a fixed photon count.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import Batch, Simulation, Sim, _check, _device_ptr, load_library
from . import wmc

__all__ = ["MLP", "features", "make_labels", "Surrogate", "BOUND"]

BOUND = [
    "mcml_mlp_create", "mcml_mlp_set_normalization", "mcml_mlp_num_params",
    "mcml_mlp_get_params", "mcml_mlp_set_params", "mcml_mlp_gradients",
    "mcml_mlp_train_epoch", "mcml_mlp_predict", "mcml_mlp_sync", "mcml_mlp_destroy",
]


class MlpConfig(C.Structure):
    _fields_ = [
        ("in_dim", C.c_int32), ("hidden", C.c_int32), ("depth", C.c_int32),
        ("out_dim", C.c_int32), ("ensemble", C.c_int32), ("seed", C.c_uint64),
        ("device", C.c_int32), ("stream", C.c_void_p),
    ]


def _bind(lib):
    if getattr(lib, "_mlp_bound", False):
        return
    vp = C.c_void_p
    sig = {
        "mcml_mlp_create": (C.c_int, [C.POINTER(MlpConfig), C.POINTER(vp)]),
        "mcml_mlp_set_normalization": (C.c_int, [vp, vp, vp, vp, vp]),
        "mcml_mlp_num_params": (C.c_int64, [vp]),
        "mcml_mlp_get_params": (C.c_int, [vp, vp, C.c_int]),
        "mcml_mlp_set_params": (C.c_int, [vp, vp, C.c_int]),
        "mcml_mlp_gradients": (C.c_int, [vp, vp, vp, C.c_int, vp, vp]),
        "mcml_mlp_train_epoch": (C.c_int, [vp, vp, vp, C.c_uint64, C.c_uint32, C.c_float,
                                           C.c_uint64, vp]),
        "mcml_mlp_predict": (C.c_int, [vp, vp, C.c_uint64, vp, vp, C.c_uint32]),
        "mcml_mlp_sync": (C.c_int, [vp]),
        "mcml_mlp_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._mlp_bound = True


class MLP:
    """Ensemble of MLPs (in -> hidden x depth, GELU -> out) on the GPU."""

    def __init__(self, in_dim: int, out_dim: int, *, hidden: int = 256, depth: int = 4,
                 ensemble: int = 4, seed: int = 0, device: int = 0, stream: Optional[int] = None):
        self.lib = load_library()
        _bind(self.lib)
        self.in_dim, self.out_dim, self.hidden, self.depth = in_dim, out_dim, hidden, depth
        self.ensemble, self.device = ensemble, device
        cfg = MlpConfig(in_dim, hidden, depth, out_dim, ensemble, seed, device, stream)
        self._h = C.c_void_p()
        _check(self.lib.mcml_mlp_create(C.byref(cfg), C.byref(self._h)), "mcml_mlp_create")
        self.num_params = int(self.lib.mcml_mlp_num_params(self._h))

    def layer_shapes(self):
        in_pad = (self.in_dim + 15) // 16 * 16
        fans = [in_pad] + [self.hidden] * self.depth + [self.out_dim]
        return list(zip(fans[:-1], fans[1:]))

    def set_normalization(self, x_mean, x_std, t_mean, t_std):
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float32))
        arrs = [f(x_mean), f(x_std), f(t_mean), f(t_std)]
        _check(self.lib.mcml_mlp_set_normalization(self._h, *[a.ctypes.data_as(C.c_void_p)
                                                               for a in arrs]),
               "mcml_mlp_set_normalization")

    def params(self, member: int = 0) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        _check(self.lib.mcml_mlp_get_params(self._h, out.ctypes.data_as(C.c_void_p), member),
               "mcml_mlp_get_params")
        return out

    def set_params(self, values, member: int = 0):
        v = np.ascontiguousarray(np.asarray(values, np.float32))
        assert v.size == self.num_params
        _check(self.lib.mcml_mlp_set_params(self._h, v.ctypes.data_as(C.c_void_p), member),
               "mcml_mlp_set_params")

    def gradients(self, X, T):
        """X: (n, in) and T: (n, out) float32 CUDA tensors -> (loss[E], grads[E, P])."""
        n = X.shape[0]
        px, pt = self._xt(X, T)
        loss = np.empty(self.ensemble, np.float32)
        grads = np.empty((self.ensemble, self.num_params), np.float32)
        _check(self.lib.mcml_mlp_gradients(self._h, px, pt, n,
                                           loss.ctypes.data_as(C.c_void_p),
                                           grads.ctypes.data_as(C.c_void_p)),
               "mcml_mlp_gradients")
        return loss, grads

    def _xt(self, X, T):
        """Checked device addresses of inputs X (n, in) and targets T (n, out)."""
        n = X.shape[0] if hasattr(X, "shape") else None
        return (_device_ptr(X, "X", device=self.device, shape=(None, self.in_dim)),
                _device_ptr(T, "T", device=self.device, shape=(n, self.out_dim)))

    def train_epoch(self, X, T, *, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
        """One epoch over X (n, in) and T (n, out), float32 CUDA tensors."""
        px, pt = self._xt(X, T)
        loss = np.empty(self.ensemble, np.float32)
        _check(self.lib.mcml_mlp_train_epoch(self._h, px, pt, X.shape[0], batch, lr,
                                             seed, loss.ctypes.data_as(C.c_void_p)),
               "mcml_mlp_train_epoch")
        return loss

    def predict(self, X, chunk: int = 0):
        """X: (n, in) float32 CUDA tensor -> (mean, spread) CUDA tensors (n, out).
        chunk: rows per step of the layer-by-layer path (0: the library default)."""
        import torch
        px = _device_ptr(X, "X", device=self.device, shape=(None, self.in_dim))
        n = X.shape[0]
        mean = torch.empty((n, self.out_dim), dtype=torch.float32, device=X.device)
        spread = torch.empty_like(mean)
        _check(self.lib.mcml_mlp_predict(self._h, px, n, C.c_void_p(mean.data_ptr()),
                                         C.c_void_p(spread.data_ptr()), chunk),
               "mcml_mlp_predict")
        _check(self.lib.mcml_mlp_sync(self._h), "mcml_mlp_sync")
        return mean, spread

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.mcml_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def features(sims: Sequence[Sim]) -> np.ndarray:
    """(height, mua, mus, n, g) per layer, the last layer's height 0."""
    rows = []
    for s in sims:
        L = int(s.num_layers)
        f = []
        for l in range(L):
            f += [float(s.height[l]) if l < L - 1 else 0.0, float(s.mua[l]), float(s.mus[l]),
                  float(s.n[l]), float(s.g[l])]
        rows.append(f)
    return np.asarray(rows, np.float32)


@dataclass
class Labels:
    X: np.ndarray          # (n, 5L) features
    logR: np.ndarray       # (n, S) log reflectance
    baselines: list        # the replayed tissues


def make_labels(base: Sim, *, n_baselines: int, photons: int, combos_per_baseline: int,
                mua_range=(0.05, 0.5), mus_range=(50.0, 250.0), mus_jitter: float = 0.05,
                mua_baseline: str = "mid", seed: int = 0, device: int = 0) -> Labels:
    """White-MC labels: n_baselines tissues (mus drawn in mus_range, mua at
    the middle of its range, or at its low end with mua_baseline="low")
    walked with `photons` photons and replayed; each replay relabelled to
    combos_per_baseline (mua', mus') with mua' uniform in mua_range and
    mus' = mus * U(1 - mus_jitter, 1 + mus_jitter) clipped to mus_range (so
    the training hull is the two ranges).  From the low end every mua'
    rescale multiplies a photon's weight by exp(-dmua PL) <= 1, so long
    paths never gain weight (no heavy-tailed rescale factors)."""
    rng = np.random.default_rng(seed)
    L, S = int(base.num_layers), int(base.num_sds)
    Xs, Ys, bl = [], [], []
    for b in range(n_baselines):
        sim = Sim.from_buffer_copy(base)
        sim.number_photons = photons
        mua0 = np.full(L, mua_range[0] if mua_baseline == "low"
                       else 0.5 * (mua_range[0] + mua_range[1]))
        mus0 = rng.uniform(*mus_range, L)
        for l in range(L):
            sim.mua[l], sim.mus[l] = float(mua0[l]), float(mus0[l])
        with Simulation(sim, seed=seed * 100003 + b, device=device) as run:
            run.run()
            run.replay()
            rows = [run.rows(s) for s in range(1, S + 1)]
        combos = np.hstack([rng.uniform(*mua_range, (combos_per_baseline, L)),
                            np.clip(mus0[None, :] * rng.uniform(1 - mus_jitter, 1 + mus_jitter,
                                                                (combos_per_baseline, L)),
                                    *mus_range)]).astype(np.float32)
        R = np.stack([wmc.rescale(r, n, sim.mua[:L], sim.mus[:L], combos, photons,
                                  device=device).cpu().numpy() for r, n in rows], axis=1)
        feats = np.repeat(features([sim]), combos_per_baseline, axis=0)
        for l in range(L):
            feats[:, 5 * l + 1] = combos[:, l]
            feats[:, 5 * l + 2] = combos[:, L + l]
        ok = np.all(R > 0, axis=1)
        Xs.append(feats[ok])
        Ys.append(np.log(R[ok]))
        bl.append(sim)
    return Labels(np.concatenate(Xs), np.concatenate(Ys).astype(np.float32), bl)


class Surrogate:
    """Trained ensemble + fallback policy.  serve() returns per-SDS
    reflectance and, per query, whether plain MC answered it."""

    def __init__(self, mlp: MLP, hull_lo: np.ndarray, hull_hi: np.ndarray, *,
                 max_spread: float = 0.05, fallback_photons: int = 10_000_000,
                 fallback_seed: int = 1):
        self.mlp, self.lo, self.hi = mlp, np.asarray(hull_lo), np.asarray(hull_hi)
        self.max_spread = max_spread
        self.fallback_photons = fallback_photons
        self.fallback_seed = fallback_seed

    @classmethod
    def train(cls, labels: Labels, *, epochs: int = 20, batch: int = 4096, lr: float = 2e-3,
              hidden: int = 256, depth: int = 4, ensemble: int = 4, seed: int = 0, device: int = 0,
              **kw):
        import torch
        X, Y = labels.X, labels.logR
        mlp = MLP(X.shape[1], Y.shape[1], hidden=hidden, depth=depth, ensemble=ensemble, seed=seed,
                  device=device)
        xs = X.std(axis=0)
        mlp.set_normalization(X.mean(axis=0), np.where(xs > 1e-6, xs, 0.0), Y.mean(axis=0),
                              Y.std(axis=0))
        dev = torch.device("cuda", device)
        Xt = torch.from_numpy(X).to(dev)
        Yt = torch.from_numpy(Y).to(dev)
        history = []
        for e in range(epochs):
            rate = lr * 0.5 * (1 + np.cos(np.pi * e / epochs))  # cosine schedule
            history.append(mlp.train_epoch(Xt, Yt, batch=batch, lr=float(rate), seed=seed + e))
        s = cls(mlp, X.min(axis=0), X.max(axis=0), **kw)
        s.history = history
        return s

    def predict(self, X: np.ndarray):
        import torch
        Xt = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(
            torch.device("cuda", self.mlp.device))
        mean, spread = self.mlp.predict(Xt)
        return mean.cpu().numpy(), spread.cpu().numpy()

    def serve(self, sims: Sequence[Sim]):
        X = features(sims)
        logR, spread = self.predict(X)
        inside = np.all((X >= self.lo - 1e-6) & (X <= self.hi + 1e-6), axis=1)
        agree = np.all(spread <= self.max_spread, axis=1)
        use_mc = ~(inside & agree)
        R = np.exp(logR).astype(np.float64)
        if use_mc.any():
            idx = np.nonzero(use_mc)[0]
            fb = []
            for i in idx:
                s = Sim.from_buffer_copy(sims[i])
                s.number_photons = self.fallback_photons
                fb.append(s)
            with Batch(fb, seed=self.fallback_seed, device=self.mlp.device) as b:
                res = b.run()
            for i, r in zip(idx, res):
                R[i] = np.array(r.reflectance[:R.shape[1]])
        return R, use_mc
