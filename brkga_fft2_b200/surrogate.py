"""Python side of the makespan surrogate (``brkga_surrogate.cu``).

``Surrogate`` owns one ``BrkgaSurrogate*``: an MLP (features -> 512 -> 256 ->
1) whose matrix products run as bf16 tcgen05 GEMMs, trained online with Adam
on (chromosome features, exact makespan) pairs that the decoder produces.
It only ranks candidates; every makespan the GA reports still comes from the
exact decoder.  The reference has no counterpart (its GA decodes every
offspring, ``BRKGA_alg3.py:119-123``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi

IO_PARAMS, IO_GRADS, IO_X, IO_Y, IO_LOSS, IO_NORM, IO_ADAM, IO_STEP = range(8)
H1, H2 = 512, 256


def split_params(flat: np.ndarray, in_pad: int):
    """Flat parameter vector -> dict (W1 [512, in_pad], b1, W2 [256, 512], b2, w3, b3)."""
    o = 0
    out = {}
    for name, shape in (("W1", (H1, in_pad)), ("b1", (H1,)), ("W2", (H2, H1)), ("b2", (H2,)), ("w3", (H2,)),
                        ("b3", (1,))):
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


FEATURES = {"decode": 0, "order": 1}  # BRKGA_SURROGATE_FEATURES_DECODE / _ORDER


class Surrogate:
    """``features``: "decode" (per part in decode order its machine, proc time
    and height time, then per machine its area and time load) or "order"
    (the parts sorted by sequencing key, per part its key, area and height)."""

    def __init__(self, native_problem, max_batch: int = 4096, buffer_capacity: int = 200_000, seed: int = 0,
                 features: str = "decode"):
        import torch
        self.torch = torch
        self.lib = abi.load_library()
        self.native_problem = native_problem  # keeps the BrkgaProblem alive
        if max_batch % 128:
            raise ValueError("max_batch must be a multiple of 128")
        if features not in FEATURES:
            raise ValueError(f"features must be one of {sorted(FEATURES)}")
        self.features_kind = features
        h = ctypes.c_void_p()
        abi.check(self.lib.brkga_surrogate_create_ex(native_problem.handle, int(max_batch), int(buffer_capacity),
                                                     ctypes.c_uint64(seed), FEATURES[features], ctypes.byref(h)),
                  "brkga_surrogate_create_ex")
        self.handle = h
        a, b, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        abi.check(self.lib.brkga_surrogate_dims(h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)))
        self.in_features, self.in_pad, self.n_params = a.value, b.value, n.value
        self.max_batch = int(max_batch)
        self.capacity = int(buffer_capacity)

    def reset(self):
        """Initial weights, empty example buffer (synchronous)."""
        abi.check(self.lib.brkga_surrogate_reset(self.handle), "brkga_surrogate_reset")

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.brkga_surrogate_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self, stream=None):
        s = stream if stream is not None else self.torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream)

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr())

    # ---- online use ----------------------------------------------------------------
    def predict(self, chrom, out=None, stream=None):
        """Predicted makespans (float64 CUDA tensor) of chromosomes chrom [P, 2N] (CUDA float32)."""
        torch = self.torch
        P = chrom.shape[0]
        if out is None:
            out = torch.empty(P, dtype=torch.float64, device=chrom.device)
        abi.check(self.lib.brkga_surrogate_predict(self.handle, self._p(chrom), P, self._p(out), self._s(stream)),
                  "brkga_surrogate_predict")
        return out

    def observe(self, chrom, makespan, stream=None):
        abi.check(self.lib.brkga_surrogate_observe(self.handle, self._p(chrom), self._p(makespan), chrom.shape[0],
                                                   self._s(stream)), "brkga_surrogate_observe")

    def train(self, steps: int, batch: int = 1024, lr: float = 1e-3, stream=None):
        abi.check(self.lib.brkga_surrogate_train(self.handle, int(steps), int(batch), ctypes.c_float(lr),
                                                 self._s(stream)), "brkga_surrogate_train")

    # ---- pieces used by tests ------------------------------------------------------
    def _io(self, what, arr: np.ndarray, to_device: bool):
        abi.check(self.lib.brkga_surrogate_io(self.handle, what, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes,
                                              int(to_device)), "brkga_surrogate_io")
        return arr

    def params(self) -> np.ndarray:
        self.torch.cuda.synchronize()
        return self._io(IO_PARAMS, np.zeros(self.n_params, np.float32), False)

    def set_params(self, flat: np.ndarray):
        self._io(IO_PARAMS, np.ascontiguousarray(flat, dtype=np.float32), True)

    def grads(self) -> np.ndarray:
        self.torch.cuda.synchronize()
        return self._io(IO_GRADS, np.zeros(self.n_params, np.float32), False)

    def loss(self) -> float:
        self.torch.cuda.synchronize()
        return float(self._io(IO_LOSS, np.zeros(1, np.float32), False)[0])

    def norm(self):
        self.torch.cuda.synchronize()
        return self._io(IO_NORM, np.zeros(3, np.float64), False)

    def features(self, chrom) -> np.ndarray:
        """Feature rows of chrom (as float32 values of the bf16 features), [P, in_pad]."""
        P = chrom.shape[0]
        abi.check(self.lib.brkga_surrogate_features(self.handle, self._p(chrom), P, self._s()))
        self.torch.cuda.synchronize()
        raw = self._io(IO_X, np.zeros(self.max_batch * self.in_pad, np.uint16), False)[:P * self.in_pad]
        return (raw.astype(np.uint32) << 16).view(np.float32).reshape(P, self.in_pad)

    def load_batch(self, X_bf16, t, n_valid):
        abi.check(self.lib.brkga_surrogate_load_batch(self.handle, self._p(X_bf16), self._p(t), X_bf16.shape[0],
                                                      int(n_valid), self._s()))

    def gradients(self, B):
        abi.check(self.lib.brkga_surrogate_gradients(self.handle, int(B), self._s()))

    def adam(self, lr):
        abi.check(self.lib.brkga_surrogate_adam(self.handle, ctypes.c_float(lr), self._s()))

    def predictions(self, B) -> np.ndarray:
        self.torch.cuda.synchronize()
        return self._io(IO_Y, np.zeros(self.max_batch, np.float32), False)[:B]


def spearman(a, b) -> float:
    """Spearman rank correlation (average ranks for ties)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size < 2:
        return float("nan")

    def ranks(x):
        order = np.argsort(x, kind="stable")
        r = np.empty(x.size, np.float64)
        r[order] = np.arange(x.size)
        _, inv, cnt = np.unique(x, return_inverse=True, return_counts=True)
        sums = np.zeros(cnt.size)
        np.add.at(sums, inv, r)
        return sums[inv] / cnt[inv]

    ra, rb = ranks(a), ranks(b)
    ra -= ra.mean()
    rb -= rb.mean()
    den = np.sqrt((ra * ra).sum() * (rb * rb).sum())
    return float((ra * rb).sum() / den) if den > 0 else float("nan")
