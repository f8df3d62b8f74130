"""The learned warm start: an MLP from case parameters to macroscopic fields.

The network (dgbgk_mlp_* in lib/libdgbgk.so) runs and trains on the GPU with
hand-written tcgen05 BF16 GEMMs accumulating in FP32, FP32 master weights
and Adam.  This module is its host side.
"""
import ctypes
from ctypes import c_double, c_float, c_void_p

import numpy as np

from ._lib import check, lib, ptr


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class MLP:
    """n_in (<= 64) -> `depth` tanh layers of `width` -> n_out (linear).

    width, n_out and batch are multiples of 128 (the GEMM tile)."""

    def __init__(self, n_in=3, width=512, depth=4, n_out=32768, batch=256, seed=0, device=0):
        h = c_void_p()
        check(lib().dgbgk_mlp_create(n_in, width, depth, n_out, batch, seed, device, ctypes.byref(h)))
        self._h = h
        self.n_in, self.width, self.depth, self.n_out, self.batch = n_in, width, depth, n_out, batch

    def close(self):
        if self._h:
            lib().dgbgk_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dims(self):
        return self.n_in, self.width, self.depth, self.n_out

    def param_count(self):
        return int(lib().dgbgk_mlp_param_count(self._h))

    def get_params(self):
        p = np.empty(self.param_count(), dtype=np.float32)
        check(lib().dgbgk_mlp_get_params(self._h, ptr(p, c_float)))
        return p

    def set_params(self, p):
        p = _f32(p)
        assert p.size == self.param_count()
        check(lib().dgbgk_mlp_set_params(self._h, ptr(p, c_float)))

    def forward(self, x):
        x = _f32(x).reshape(-1, self.n_in)
        y = np.empty((x.shape[0], self.n_out), dtype=np.float32)
        check(lib().dgbgk_mlp_forward(self._h, ptr(x, c_float), x.shape[0], ptr(y, c_float)))
        return y

    def gradient(self, x, t):
        """(loss, flat gradient) of one batch of exactly `batch` rows."""
        x, t = _f32(x).reshape(-1, self.n_in), _f32(t).reshape(-1, self.n_out)
        loss = c_double()
        g = np.empty(self.param_count(), dtype=np.float32)
        check(lib().dgbgk_mlp_gradient(self._h, ptr(x, c_float), ptr(t, c_float), x.shape[0], ctypes.byref(loss),
                                       ptr(g, c_float)))
        return loss.value, g

    def set_data(self, x, t):
        x, t = _f32(x).reshape(-1, self.n_in), _f32(t).reshape(-1, self.n_out)
        assert x.shape[0] == t.shape[0]
        check(lib().dgbgk_mlp_set_data(self._h, ptr(x, c_float), ptr(t, c_float), x.shape[0]))

    def train(self, iters, lr=1e-3, seed=0):
        """`iters` Adam steps on the training set; returns each step's loss."""
        hist = np.zeros(iters)
        check(lib().dgbgk_mlp_train(self._h, iters, lr, seed, ptr(hist)))
        return hist


def main(argv=None):
    """Training throughput of the network on synthetic data:

        python -m dgbgk.warmstart --batch 1024 --iters 50

    prints the Adam steps per second and the tensor-core FLOP rate of the
    GEMMs (6 * batch * sum of layer in*out FLOPs per step: forward, and the
    weight and input gradients)."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="warm-start network training throughput")
    ap.add_argument("--width", type=int, default=512)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--n-out", type=int, default=32768)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)
    m = MLP(3, a.width, a.depth, a.n_out, a.batch, seed=0)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (4 * a.batch, 3)).astype(np.float32)
    t = rng.normal(0, 1, (4 * a.batch, a.n_out)).astype(np.float32)
    m.set_data(x, t)
    m.train(a.warmup, lr=1e-4)
    t0 = time.perf_counter()
    m.train(a.iters, lr=1e-4)
    dt = time.perf_counter() - t0
    layers = [(64, a.width)] + [(a.width, a.width)] * (a.depth - 1) + [(a.width, a.n_out)]
    flops = 6.0 * a.batch * sum(i * o for i, o in layers) * a.iters
    print(json.dumps({"batch": a.batch, "params": m.param_count(), "iters": a.iters, "ms_per_iter": 1e3 * dt / a.iters,
                      "gemm_tflops": flops / dt / 1e12}))
    m.close()


if __name__ == "__main__":
    main()
