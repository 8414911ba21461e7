"""The surrogate network of the delayed-acceptance Monte Carlo on the device.

``SurrogateNet`` holds a 1280 -> 128 -> 128 -> 1 perceptron (SiLU, BF16 weights and
activations, FP32 accumulation) as device tensors and drives the library's tcgen05 kernels:
``forward`` evaluates rows of BF16 features, ``train_step`` takes one Adam step on a batch of
row pairs (the features of a move in both orders) whose antisymmetric output is fitted to
the move's energy change.  The network is this project's addition; the reference method has
no counterpart.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

IN, H = 1280, 128
NPARAM = H * IN + H + H * H + H + H + 1


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class SurrogateNet:
    def __init__(self, device="cuda", seed=0, params=None):
        self.lib = _lib.load(require_device=True)
        self.dev = torch.device(device)
        if params is None:
            rng = np.random.default_rng(seed)
            params = dict(w1=rng.standard_normal((H, IN)) / np.sqrt(IN), b1=np.zeros(H),
                          w2=rng.standard_normal((H, H)) / np.sqrt(H), b2=np.zeros(H),
                          w3=rng.standard_normal(H) / np.sqrt(H), b3=np.zeros(1))
        f = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev)  # noqa: E731
        self.w1, self.b1, self.w2 = f(params["w1"]), f(params["b1"]), f(params["w2"])
        self.b2, self.w3, self.b3 = f(params["b2"]), f(params["w3"]), f(params["b3"])
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)  # noqa: E731
        self.w1h = torch.zeros(H, IN, dtype=torch.bfloat16, device=self.dev)
        self.w2h = torch.zeros(H, H, dtype=torch.bfloat16, device=self.dev)
        self.w2th = torch.zeros(H, H, dtype=torch.bfloat16, device=self.dev)
        self.dw1, self.db1, self.dw2, self.db2, self.dw3, self.db3 = z(H, IN), z(H), z(H, H), z(H), z(H), z(1)
        self.m1, self.v1 = z(NPARAM), z(NPARAM)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        n = _lib.Mlp()
        for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w1h", "w2h", "w2th", "dw1", "db1", "dw2", "db2", "dw3", "db3",
                  "m1", "v1", "status"):
            setattr(n, k, _p(getattr(self, k)))
        self.c = n
        self.step = 0
        self._work = None
        check(self.lib.epsr_mlp_sync_weights(C.byref(self.c), _stream()))

    def params(self):
        return {k: getattr(self, k).cpu().numpy().copy() for k in ("w1", "b1", "w2", "b2", "w3", "b3")}

    def work(self, rows):
        nb = int(self.lib.epsr_mlp_work_bytes(int(rows)))
        if self._work is None or self._work.numel() < nb:
            self._work = torch.empty(nb, dtype=torch.uint8, device=self.dev)
        return self._work

    def forward(self, x, y=None):
        """y[r] for x [rows][1280] BF16 (a device tensor)."""
        rows = x.shape[0]
        if y is None:
            y = torch.empty(rows, dtype=torch.float32, device=self.dev)
        w = self.work(rows)
        check(self.lib.epsr_mlp_forward(C.byref(self.c), _p(x), rows, _p(y), _p(w), w.numel(), _stream()))
        return y

    def train_step(self, x, xt, row0, rows, target, lr, loss=None):
        """One Adam step on rows row0..row0+rows-1 of x (xt = x transposed, [1280][ld])."""
        self.step += 1
        w = self.work(rows)
        check(self.lib.epsr_mlp_train_step(C.byref(self.c), _p(x), _p(xt), xt.shape[1], int(row0), int(rows),
                                           _p(target), float(lr), self.step, _p(loss), _p(w), w.numel(), _stream()))

    def check_status(self):
        if int(self.status.item()):
            raise _lib.EpsrGpuError(5, "surrogate kernel: a bounded wait gave up")


def umma_gemm(a, b, kslices=1, accumulate=False, out=None):
    """D = a . b^T on the tensor cores (a [m][k], b [n][k] BF16 device tensors), FP32."""
    lib = _lib.load(require_device=True)
    m, k = a.shape
    n = b.shape[0]
    if out is None:
        out = torch.zeros(m, n, dtype=torch.float32, device=a.device)
    st = torch.zeros(1, dtype=torch.int32, device=a.device)
    check(lib.epsr_umma_gemm_f32(_p(a), m, _p(b), n, k, kslices, _p(out), out.shape[1], 1 if accumulate else 0,
                                 _p(st), _stream()))
    if int(st.item()):
        raise _lib.EpsrGpuError(5, "umma gemm: a bounded wait gave up")
    return out
