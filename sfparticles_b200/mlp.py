"""Learned photon-energy sampler for the optical-depth method.

This has no counterpart in the reference. When photon emission occurs, the
optical-depth method draws the photon's energy fraction δ from an inverse-CDF
table: ``_bisect_interp`` (``qed/optical_depth_tables.py:59-102``), a
bisection over 1024 δ nodes between two χ rows. ``PhotonSampler`` replaces that
bisection with a small network, (log10 χ, u) → δ:

- architecture: 2 → 64 → 64 → 64 → 1 with SiLU, 8577 parameters; the inputs
  are log10 χ / 3 and logit(u) / 8, and the output is log10 δ / 3 + 1;
- trained on samples that the method's own table generates;
- inference on the tensor cores (BF16 weights, FP32 accumulation);
- training by this package's own kernels: a fused forward/backward pass and
  Adam.

The table sampler stays available: ``sample_table`` is the batched reference
the network is trained on and judged against.

Typical use::

    s = PhotonSampler.trained()          # committed weights, or train here
    delta = s.sample(log_chi, u)         # torch float64 tensors on the GPU
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from . import _lib

H = 64
NPARAM = 8577
# parameter layout: W0[64][2] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[64] b3
OFFSETS = {"W0": (0, (H, 2)), "b0": (128, (H,)), "W1": (192, (H, H)), "b1": (4288, (H,)), "W2": (4352, (H, H)),
           "b2": (8448, (H,)), "W3": (8512, (H,)), "b3": (8576, ())}
WEIGHTS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qed", "data", "mlp_photon.npy")
LOG_CHI_RANGE = (-3.0, 3.0)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    fan = {"W0": 2, "b0": 2, "W1": H, "b1": H, "W2": H, "b2": H, "W3": H, "b3": H}
    for k, (off, shape) in OFFSETS.items():
        n = int(np.prod(shape)) if shape else 1
        b = 1.0 / math.sqrt(fan[k])
        p[off:off + n] = rng.uniform(-b, b, n)
    return p


def _photon_table():
    from .particles import _device
    from .qed import device_tables
    return device_tables.od_tables(_device())[0]


def sample_table(log_chi, u):
    """The optical-depth photon table sampler, batched: δ for each (log10 χ, u)
    (float64 CUDA tensors)."""
    import torch
    log_chi = log_chi.contiguous()
    u = u.contiguous()
    out = torch.empty_like(log_chi, dtype=torch.float64)
    tab = _photon_table()
    _lib.call("sfp_od_inverse_cdf", ctypes.byref(tab), _p(log_chi), _p(u), _p(out), log_chi.numel(), _stream())
    return out


class PhotonSampler(object):
    def __init__(self, params=None):
        import torch
        from .particles import _device
        p = init_params() if params is None else np.asarray(params, dtype=np.float32)
        if p.shape != (NPARAM,):
            raise ValueError(f"expected {NPARAM} parameters, got {p.shape}")
        self.params = torch.as_tensor(p, device=_device()).contiguous()
        self.losses = []

    # -------------------------------------------------------------- I/O
    @classmethod
    def load(cls, path: str = WEIGHTS_FILE) -> "PhotonSampler":
        return cls(np.load(path))

    def save(self, path: str = WEIGHTS_FILE) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.save(path, self.params.cpu().numpy())

    @classmethod
    def trained(cls, **train_kw) -> "PhotonSampler":
        """The committed trained weights, or a network trained here on the GPU."""
        if os.path.exists(WEIGHTS_FILE):
            return cls.load()
        s = cls()
        s.train(**train_kw)
        return s

    # --------------------------------------------------------- inference
    def sample(self, log_chi, u, kernel: str = "tcgen05"):
        """δ for each (log10 χ, u), float64 CUDA tensors, on the tensor cores:
        kernel 'tcgen05' (128-query tiles, accumulators in tensor memory) or
        'warp' (the step's warp-level mma.sync tiles of 16 queries)."""
        import torch
        log_chi = log_chi.contiguous()
        u = u.contiguous()
        out = torch.empty_like(log_chi, dtype=torch.float64)
        fn = {"tcgen05": "sfp_mlp_infer", "warp": "sfp_mlp_infer_warp"}[kernel]
        _lib.call(fn, _p(self.params), _p(log_chi), _p(u), _p(out), log_chi.numel(), _stream())
        return out

    @staticmethod
    def device_error() -> int:
        """1 if a tcgen05 inference launch gave up waiting for its tensor
        cores since the last call (synchronises the device), else 0."""
        code = ctypes.c_int(0)
        _lib.call("sfp_mlp_device_error", ctypes.byref(code))
        return int(code.value)

    # ---------------------------------------------------------- training
    @staticmethod
    def make_samples(n: int, seed: int = 1, chunk: int = 0, log_chi_range=LOG_CHI_RANGE):
        """n training samples from the table: (features [n, 2], targets [n]) float32."""
        import torch
        from .particles import _device
        feat = torch.empty((n, 2), dtype=torch.float32, device=_device())
        targ = torch.empty(n, dtype=torch.float32, device=_device())
        tab = _photon_table()
        _lib.call("sfp_mlp_make_samples", ctypes.byref(tab), int(seed), int(chunk), float(log_chi_range[0]),
                  float(log_chi_range[1]), n, _p(feat), _p(targ), _stream())
        return feat, targ

    def grad(self, features, targets):
        """(gradient [8577] of Σ (y - target)², that sum): one fused forward +
        backward pass of this package's training kernel."""
        import torch
        g = torch.zeros(NPARAM, dtype=torch.float32, device=self.params.device)
        loss = torch.zeros(1, dtype=torch.float64, device=self.params.device)
        _lib.call("sfp_mlp_grad", _p(self.params), _p(features.contiguous()), _p(targets.contiguous()),
                  targets.numel(), _p(g), _p(loss), _stream())
        return g, float(loss.item())

    def train(self, n_samples: int = 100_000_000, batch: int = 65536, epochs: int = 8, lr: float = 3e-3,
              lr_end: float = 3e-5, seed: int = 1, report_every: int = 200, log=None):
        """Adam on the mean squared error of log10 δ / 3, with a cosine learning
        rate from `lr` to `lr_end`.  The n_samples training samples come from the
        table and are drawn once; each epoch visits them in order."""
        import torch
        feat, targ = self.make_samples(n_samples, seed=seed)
        dev = self.params.device
        g = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
        m = torch.zeros_like(g)
        v = torch.zeros_like(g)
        loss = torch.zeros(1, dtype=torch.float64, device=dev)
        L = _lib.load()
        nb = (n_samples + batch - 1) // batch
        total = nb * epochs
        step = 0
        run_loss, run_n = 0.0, 0
        s = _stream()
        for ep in range(epochs):
            for b in range(nb):
                lo = b * batch
                n = min(batch, n_samples - lo)
                g.zero_()
                _lib.check(L.sfp_mlp_grad(_p(self.params), ctypes.c_void_p(feat.data_ptr() + lo * 8),
                                          ctypes.c_void_p(targ.data_ptr() + lo * 4), n, _p(g), _p(loss), s),
                           "sfp_mlp_grad")
                step += 1
                rate = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * step / total))
                _lib.check(L.sfp_mlp_adam(_p(self.params), _p(g), _p(m), _p(v), step, rate, 0.9, 0.999, 1e-8,
                                          1.0 / n, s), "sfp_mlp_adam")
                run_n += n
                if step % report_every == 0 or step == total:
                    tot = float(loss.item())
                    loss.zero_()
                    self.losses.append((step, tot / max(run_n, 1)))
                    if log:
                        log(f"epoch {ep} step {step}/{total} mse {tot / max(run_n, 1):.3e} lr {rate:.2e}")
                    run_loss, run_n = 0.0, 0
        del feat, targ
        return self.losses
