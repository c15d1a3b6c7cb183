"""MLP surrogate of a scalar UQ observable on BF16 tensor cores.

Python face of ``include/als_surrogate.h``: the network is trained and
evaluated by the library's own tcgen05 kernels (forward, backward, Adam);
there is no other implementation behind this class.  Inputs and outputs are
device tensors (torch, FP32); the target is standardised on the host before
training and predictions are mapped back.
"""
import ctypes

import numpy as np

from . import _lib


class Surrogate:
    """inputs -> width (GELU) x hidden -> 1.

    The defaults are the Kelvin-Helmholtz control variate: 40 perturbation
    parameters, four hidden layers of 256 (208,129 parameters)."""

    def __init__(self, inputs=40, width=256, hidden=4, max_batch=1024, device=0, seed=0):
        import torch
        self._torch = torch
        self._lib = _lib.load()
        cfg = _lib.MlpConfig(inputs, width, hidden, max_batch)
        h = ctypes.c_void_p()
        _lib.check(self._lib.als_mlp_create(ctypes.byref(cfg), device, ctypes.byref(h)))
        self._h = h
        self.inputs, self.width, self.hidden, self.max_batch = inputs, width, hidden, max_batch
        self.device = torch.device("cuda", device)
        n = ctypes.c_longlong()
        _lib.check(self._lib.als_mlp_param_count(self._h, ctypes.byref(n)))
        self.param_count = n.value
        self.y_shift = 0.0
        self.y_scale = 1.0
        self.init(seed)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.als_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init(self, seed=0):
        _lib.check(self._lib.als_mlp_init(self._h, int(seed)))

    def params(self):
        out = np.zeros(self.param_count, dtype=np.float32)
        _lib.check(self._lib.als_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.param_count:
            raise ValueError("expected %d parameters" % self.param_count)
        _lib.check(self._lib.als_mlp_set_params(self._h, p.ctypes.data))

    def _dev(self, a, shape=None):
        torch = self._torch
        t = torch.as_tensor(a, dtype=torch.float32, device=self.device).contiguous()
        if shape is not None:
            t = t.reshape(shape)
        return t

    def forward_raw(self, x, per_layer=False):
        """Network output for rows of x (no target scaling); `per_layer`
        runs one kernel per layer instead of the whole-network kernel (the
        same results)."""
        x = self._dev(x)
        rows = x.shape[0]
        y = self._torch.empty(rows, dtype=self._torch.float32, device=self.device)
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        fn = self._lib.als_mlp_forward_layers if per_layer else self._lib.als_mlp_forward
        _lib.check(fn(self._h, x.data_ptr(), rows, y.data_ptr(), stream))
        return y

    def __call__(self, x):
        """Surrogate prediction of the observable (target scaling undone)."""
        return self.forward_raw(x) * self.y_scale + self.y_shift

    def gradients(self, x, t):
        x = self._dev(x)
        t = self._dev(t)
        g = self._torch.empty(self.param_count, dtype=self._torch.float32, device=self.device)
        loss = ctypes.c_float()
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.als_mlp_gradients(self._h, x.data_ptr(), t.data_ptr(), x.shape[0],
                                               g.data_ptr(), ctypes.byref(loss), stream))
        return g, loss.value

    def train_raw(self, x, t, steps, lr=1e-3):
        """Full-batch Adam on (x, t) as given; returns the loss of every step."""
        x = self._dev(x)
        t = self._dev(t)
        loss = self._torch.zeros(max(steps, 1), dtype=self._torch.float32, device=self.device)
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.als_mlp_train(self._h, x.data_ptr(), t.data_ptr(), x.shape[0],
                                           int(steps), float(lr), loss.data_ptr(), stream))
        return loss[:steps].cpu().numpy()

    def fit(self, params, y, steps=2000, lr=1e-3, validation=None, check_every=100):
        """Trains on (parameters, observables) with the target standardised.

        With ``validation = (params_v, y_v)`` the validation error is checked
        every ``check_every`` steps and the parameters with the lowest one are
        kept (early stopping); ``self.best_step`` records which.  Returns the
        training loss of every step."""
        y = np.asarray(y, dtype=np.float64)
        self.y_shift = float(y.mean())
        self.y_scale = float(y.std()) or 1.0
        t = (y - self.y_shift) / self.y_scale
        if validation is None:
            self.best_step = steps
            return self.train_raw(params, t, steps, lr)
        pv = self._dev(validation[0])
        yv = np.asarray(validation[1], dtype=np.float64)
        best = (np.mean((self(pv).double().cpu().numpy() - yv) ** 2), 0, self.params())
        losses = []
        done = 0
        while done < steps:
            k = min(check_every, steps - done)
            losses.append(self.train_raw(params, t, k, lr))
            done += k
            err = np.mean((self(pv).double().cpu().numpy() - yv) ** 2)
            if err < best[0]:
                best = (err, done, self.params())
        # restore the best parameters; their Adam state is not needed afterwards
        self.set_params(best[2])
        self.best_step = best[1]
        return np.concatenate(losses)

    def moments(self, samples, seed=1, chunk=1 << 20):
        """E[f] and E[f^2] over U[0,1)^inputs from `samples` device draws (FP64 sums)."""
        torch = self._torch
        s1 = torch.zeros((), dtype=torch.float64, device=self.device)
        s2 = torch.zeros((), dtype=torch.float64, device=self.device)
        x = torch.empty(chunk * self.inputs, dtype=torch.float32, device=self.device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        done = 0
        k = 0
        while done < samples:
            n = min(chunk, samples - done)
            _lib.check(self._lib.als_mlp_sample_uniform(x.data_ptr(), n * self.inputs,
                                                        int(seed) * 1000003 + k, stream))
            f = self(x[:n * self.inputs].view(n, self.inputs)).double()
            s1 += f.sum()
            s2 += (f * f).sum()
            done += n
            k += 1
        return float(s1) / samples, float(s2) / samples
