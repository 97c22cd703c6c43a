"""The learned 3D CNN of the pressure solver (include/msbg_cnn.h), from Python.

Device tensors are torch CUDA tensors (torch provides the device memory; all
compute is in libmsbg_gpu.so).  Training runs entirely on the GPU with the
library's own forward, backward and Adam kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import MsbgError, lib

NFEAT, NPAD, NCELL = 4, 18 ** 3, 16 ** 3


def _sigs(L):
    vp, i32 = C.c_void_p, C.c_int
    sig = {
        "msbg_cnn_num_params": (i32, []),
        "msbg_cnn_create": (i32, [i32, C.POINTER(vp)]),
        "msbg_cnn_destroy": (i32, [vp]),
        "msbg_cnn_last_error": (C.c_char_p, [vp]),
        "msbg_cnn_set_weights": (i32, [vp, C.POINTER(C.c_float), C.c_int64]),
        "msbg_cnn_get_weights": (i32, [vp, C.POINTER(C.c_float), C.c_int64]),
        "msbg_cnn_forward": (i32, [vp, vp, vp, i32]),
        "msbg_cnn_loss_grad": (i32, [vp, vp, vp, vp, i32, C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_float)]),
        "msbg_cnn_adam_step": (i32, [vp, C.c_float, C.c_float, C.c_float, C.c_float]),
        "msbg_gpu_pressure_set_cnn": (i32, [vp, vp]),
        "msbg_gpu_pressure_training_pairs": (i32, [vp, vp, vp, vp, i32, C.POINTER(C.c_int)]),
        "msbg_gpu_pressure_learned_guess": (i32, [vp, C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_pressure_set_correction_cnn": (i32, [vp, vp]),
        "msbg_gpu_pressure_correction_pairs": (i32, [vp, vp, i32, vp, vp, vp, i32,
                                                     C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _ptr(t):
    assert t.is_cuda and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


class Cnn:
    """One network on a device (msbg_cnn_*)."""

    def __init__(self, device=0):
        self._L = lib()
        _sigs(self._L)
        self._h = C.c_void_p()
        rc = self._L.msbg_cnn_create(device, C.byref(self._h))
        if rc:
            raise MsbgError(rc, "msbg_cnn_create")
        self.n_params = self._L.msbg_cnn_num_params()

    def _check(self, rc, what):
        if rc:
            raise MsbgError(rc, f"{what}: {self._L.msbg_cnn_last_error(self._h).decode()}")

    def close(self):
        if self._h:
            self._L.msbg_cnn_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_weights(self):
        w = np.zeros(self.n_params, np.float32)
        self._check(self._L.msbg_cnn_get_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float)),
                                                 self.n_params), "get_weights")
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self._L.msbg_cnn_set_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float)),
                                                 w.size), "set_weights")

    def forward(self, feat):
        import torch
        n = feat.shape[0]
        out = torch.empty((n, NCELL), dtype=torch.float32, device=feat.device)
        self._check(self._L.msbg_cnn_forward(self._h, _ptr(feat), _ptr(out), n), "forward")
        return out

    def loss_grad(self, feat, target, mask, count=None, want_grad=False):
        n = feat.shape[0]
        if count is None:
            count = float(mask.sum().item())
        loss = C.c_double()
        g = np.zeros(self.n_params, np.float32) if want_grad else None
        gp = g.ctypes.data_as(C.POINTER(C.c_float)) if want_grad else None
        self._check(self._L.msbg_cnn_loss_grad(self._h, _ptr(feat), _ptr(target), _ptr(mask), n,
                                               float(count), C.byref(loss), gp), "loss_grad")
        return (loss.value, g) if want_grad else loss.value

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self._check(self._L.msbg_cnn_adam_step(self._h, lr, beta1, beta2, eps), "adam_step")


def collect_training_pairs(ctx, max_pairs):
    """Pairs of the last refined solve of ctx: (feat, target, mask) torch CUDA tensors."""
    import torch
    L = lib()
    _sigs(L)
    dev = torch.device("cuda", ctx.device)
    feat = torch.zeros((max_pairs, NFEAT * NPAD), dtype=torch.float32, device=dev)
    target = torch.zeros((max_pairs, NCELL), dtype=torch.float32, device=dev)
    mask = torch.zeros((max_pairs, NCELL), dtype=torch.float32, device=dev)
    n = C.c_int()
    ctx._check(L.msbg_gpu_pressure_training_pairs(ctx._h, _ptr(feat), _ptr(target), _ptr(mask),
                                                  max_pairs, C.byref(n)), "training_pairs")
    n = n.value
    return feat[:n].contiguous(), target[:n].contiguous(), mask[:n].contiguous()


def collect_correction_pairs(ctx, max_pairs, pcg_iters, params=None, **kw):
    """Pairs of the correction network (see msbg_gpu_pressure_correction_pairs):
    the residual the V-cycle leaves after `pcg_iters` PCG iterations and the
    error it leaves, from the last refined solve of ctx."""
    import torch
    from . import solve_params
    L = lib()
    _sigs(L)
    p = params or solve_params(**kw)
    dev = torch.device("cuda", ctx.device)
    feat = torch.zeros((max_pairs, NFEAT * NPAD), dtype=torch.float32, device=dev)
    target = torch.zeros((max_pairs, NCELL), dtype=torch.float32, device=dev)
    mask = torch.zeros((max_pairs, NCELL), dtype=torch.float32, device=dev)
    n = C.c_int()
    ctx._check(L.msbg_gpu_pressure_correction_pairs(ctx._h, C.byref(p), pcg_iters, _ptr(feat),
                                                    _ptr(target), _ptr(mask), max_pairs,
                                                    C.byref(n)), "correction_pairs")
    n = n.value
    return feat[:n].contiguous(), target[:n].contiguous(), mask[:n].contiguous()


def train_cnn(net, feat, target, mask, epochs=40, batch=128, lr=2e-3, seed=0, log=None):
    """Adam on mini-batches of tiles (fixed seed); returns the loss per epoch.

    The loss of a batch is normalised by its liquid-cell count."""
    import torch
    n = feat.shape[0]
    g = torch.Generator().manual_seed(seed)
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(feat.device)
        tot, cnt = 0.0, 0
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            fb, tb, mb = feat[idx].contiguous(), target[idx].contiguous(), mask[idx].contiguous()
            c = float(mb.sum().item())
            if c <= 0:
                continue
            loss = net.loss_grad(fb, tb, mb, count=c)
            net.adam_step(lr)
            tot += loss * c
            cnt += c
        losses.append(tot / max(cnt, 1.0))
        if log:
            log(ep, losses[-1])
    return losses


def _ctx_set_cnn(self, net):
    L = lib()
    _sigs(L)
    self._check(L.msbg_gpu_pressure_set_cnn(self._h, net._h if net is not None else None),
                "set_cnn")
    self._cnn = net  # keep it alive while attached


def _ctx_set_correction_cnn(self, net):
    L = lib()
    _sigs(L)
    self._check(L.msbg_gpu_pressure_set_correction_cnn(self._h, net._h if net is not None else None),
                "set_correction_cnn")
    self._cnn_corr = net


def _ctx_learned_guess(self):
    """The attached network's pressure prediction (packed layout, FP32)."""
    L = lib()
    _sigs(L)
    n = C.c_int64()
    self._check(L.msbg_gpu_pressure_packed_size(self._h, C.byref(n)), "packed_size")
    out = np.zeros(n.value, np.float32)
    self._check(L.msbg_gpu_pressure_learned_guess(self._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                  n.value), "learned_guess")
    return out


def _install():
    from . import Context
    Context.pressure_set_cnn = _ctx_set_cnn
    Context.pressure_set_correction_cnn = _ctx_set_correction_cnn
    Context.pressure_learned_guess = _ctx_learned_guess


_install()
