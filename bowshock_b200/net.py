"""Host mirror of the warm-start network of the CUDA library (bowshock_net_*, include/bowshock_b200.h): a conv decoder of
about 1.84 M parameters whose every contraction, forward and backward, is a BF16 tcgen05 GEMM with FP32 accumulation,
trained by Adam on FP32 master weights. No counterpart in the reference (it has no learned component)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from ._ffi import BowshockError

NET_IN, NET_OUT, NET_OUT_PAD, NET_CELLS = 16, 6, 16, 2048
H_OUT, W_OUT = 32, 64
SLOPE = 0.1


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Net:
    def __init__(self, max_batch: int = 64, device: int = 0):
        h = C.c_void_p()
        rc = _ffi.load().bowshock_net_create(int(device), int(max_batch), C.byref(h))
        if rc:
            raise BowshockError(rc, "bowshock_net_create failed")
        self._h = h
        self.max_batch = max_batch
        n = C.c_uint64()
        self._check(_ffi.load().bowshock_net_num_params(self._h, C.byref(n)))
        self.nparams = n.value

    def __del__(self):
        if getattr(self, "_h", None):
            _ffi.load().bowshock_net_destroy(self._h)
            self._h = None

    def _check(self, rc):
        if rc:
            raise BowshockError(rc, (_ffi.load().bowshock_net_last_error(self._h) or b"").decode())

    def layout(self):
        """[(fc, cin, cout, H, W, up, act, woff, boff)] per layer."""
        n = C.c_uint64()
        self._check(_ffi.load().bowshock_net_layout(self._h, None, 0, C.byref(n)))
        out = np.zeros(9 * n.value, dtype=np.int64)
        self._check(_ffi.load().bowshock_net_layout(self._h, out.ctypes.data_as(C.POINTER(C.c_int64)), out.size, C.byref(n)))
        return [tuple(int(v) for v in out[9 * k:9 * k + 9]) for k in range(n.value)]

    def set_params(self, p):
        p = _f(p)
        assert p.size == self.nparams
        self._check(_ffi.load().bowshock_net_set_params(self._h, _ffi.fptr(p)))

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        self._check(_ffi.load().bowshock_net_get_params(self._h, _ffi.fptr(p)))
        return p

    def set_mask(self, mask):
        m = np.ascontiguousarray(np.asarray(mask).reshape(-1) != 0, dtype=np.uint8)
        assert m.size == NET_CELLS
        self._check(_ffi.load().bowshock_net_set_mask(self._h, m.ctypes.data_as(C.POINTER(C.c_uint8))))

    def forward(self, x) -> np.ndarray:
        """x [B, 16] -> [B, 32, 64, 6]"""
        x = _f(x).reshape(-1, NET_IN)
        y = np.zeros((x.shape[0], NET_CELLS, NET_OUT), dtype=np.float32)
        self._check(_ffi.load().bowshock_net_forward(self._h, x.shape[0], _ffi.fptr(x), _ffi.fptr(y)))
        return y.reshape(-1, H_OUT, W_OUT, NET_OUT)

    def gradients(self, x, target):
        x = _f(x).reshape(-1, NET_IN)
        t = _f(target).reshape(x.shape[0], -1)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double()
        self._check(_ffi.load().bowshock_net_gradients(self._h, x.shape[0], _ffi.fptr(x), _ffi.fptr(t), _ffi.fptr(g), C.byref(loss)))
        return loss.value, g

    def set_dataset(self, x, target):
        x = _f(x).reshape(-1, NET_IN)
        t = _f(target).reshape(x.shape[0], -1)
        assert t.shape[1] == NET_CELLS * NET_OUT
        self._check(_ffi.load().bowshock_net_set_dataset(self._h, x.shape[0], _ffi.fptr(x), _ffi.fptr(t)))

    def reset_optimizer(self):
        self._check(_ffi.load().bowshock_net_reset_optimizer(self._h))

    def train(self, steps: int, batch: int, lr: float, seed: int = 0) -> np.ndarray:
        loss = np.zeros(steps)
        self._check(_ffi.load().bowshock_net_train(self._h, int(steps), int(batch), float(lr), int(seed), _ffi.dptr(loss)))
        return loss

    CONV_IM2COL, CONV_GATHER, CONV_TMA = 0, 1, 2

    def set_conv_mode(self, mode: int):
        """3x3 convolutions as implicit GEMMs fed by TMA boxes (CONV_TMA, the default), as implicit GEMMs gathered by
        cp.async (CONV_GATHER), or through an im2col matrix (CONV_IM2COL)."""
        self._check(_ffi.load().bowshock_net_set_conv_mode(self._h, int(mode)))

    def last_train_ms(self) -> float:
        ms = C.c_double()
        self._check(_ffi.load().bowshock_net_last_train_ms(self._h, C.byref(ms)))
        return ms.value


def flops_per_sample(layout) -> float:
    """Forward multiply-add FLOPs of one sample: 2 x sum over layers of cout x kin x output pixels."""
    total = 0.0
    for fc, cin, cout, H, W, up, act, woff, boff in layout:
        total += 2.0 * cout * (cin if fc else 9 * cin) * (1 if fc else H * W)
    return total
