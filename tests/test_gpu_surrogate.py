"""The BF16 tensor-core MLP surrogate on the GPU, against the CPU oracle.

Forward outputs and MSE gradients of the tcgen05 kernels are compared with
oracle/mlp_oracle.py, which rounds to BF16 at the same points; what is left
is FP32 accumulation order and the odd BF16 rounding flip, hence relative
tolerances of 1e-2 (stated per test).  Training, Adam and inference in
chunks are checked for their own invariants, and the control variate built
from a trained network is shown to cut the variance of the Monte Carlo
estimator on solver-generated Kelvin-Helmholtz samples.
"""
import os
import sys

import numpy as np
import pytest
import torch

import alsvinn_b200 as als
from conftest import ROOT, load_golden

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def _blocks(flat, inputs, width, hidden):
    out = []
    off = 0
    for o, i in mo.layer_shapes(inputs, width, hidden):
        out.append(("W%d" % len(out), flat[off:off + o * i]))
        off += o * i
        out.append(("b%d" % (len(out) // 2), flat[off:off + o]))
        off += o
    return out


@pytest.mark.parametrize("inputs,width,hidden,rows", [(40, 256, 4, 300), (7, 64, 2, 128),
                                                      (40, 128, 3, 1000)])
def test_forward_matches_oracle(inputs, width, hidden, rows):
    rng = np.random.default_rng(rows + width)
    x = rng.uniform(0, 1, (rows, inputs)).astype(np.float32)
    with als.Surrogate(inputs, width, hidden, max_batch=1024, seed=11) as s:
        y = s.forward_raw(x).cpu().numpy().astype(np.float64)
        p = s.params()
    ref, _ = mo.forward(p, x, inputs, width, hidden, bf16_path=True)
    scale = np.abs(ref).max() + 1e-3
    # FP32 accumulation vs FP64, occasional BF16 rounding flips: 1e-2 of the output scale
    assert np.abs(y - ref).max() <= 1e-2 * scale, np.abs(y - ref).max()
    # and a close match on average
    assert np.abs(y - ref).mean() <= 1e-3 * scale


@pytest.mark.parametrize("rows", [256, 200])
def test_gradients_match_oracle(rows):
    inputs, width, hidden = 40, 256, 4
    rng = np.random.default_rng(rows)
    x = rng.uniform(0, 1, (rows, inputs)).astype(np.float32)
    t = rng.normal(0, 1, rows).astype(np.float32)
    with als.Surrogate(inputs, width, hidden, max_batch=1024, seed=5) as s:
        g, loss = s.gradients(x, t)
        g = g.cpu().numpy().astype(np.float64)
        p = s.params()
    ref, ref_loss = mo.gradients(p, x, t, inputs, width, hidden, bf16_path=True)
    assert loss == pytest.approx(ref_loss, rel=1e-3)
    for (name, a), (_, b) in zip(_blocks(g, inputs, width, hidden),
                                 _blocks(ref, inputs, width, hidden)):
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        # relative error of each parameter block's gradient: 1e-2
        assert rel < 1e-2, (name, rel)
    cos = np.dot(g, ref) / (np.linalg.norm(g) * np.linalg.norm(ref))
    assert cos > 0.9999


def test_first_adam_step_moves_every_parameter_by_lr():
    inputs, width, hidden, rows = 40, 256, 4, 512
    rng = np.random.default_rng(9)
    x = rng.uniform(0, 1, (rows, inputs)).astype(np.float32)
    t = rng.normal(0, 1, rows).astype(np.float32)
    lr = 1e-3
    with als.Surrogate(inputs, width, hidden, max_batch=1024, seed=2) as s:
        p0 = s.params()
        g, _ = s.gradients(x, t)
        g = g.cpu().numpy()
        s.train_raw(x, t, 1, lr)
        p1 = s.params()
    # first Adam step: m_hat = g, v_hat = g^2 -> p - lr * g / (|g| + eps)
    expected = p0.astype(np.float64) - lr * g / (np.abs(g) + 1e-8)
    assert np.abs(p1 - expected).max() <= 1e-6


def test_training_reduces_the_loss():
    inputs, width, hidden, rows = 40, 256, 4, 1024
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, (rows, inputs))
    a = rng.normal(0, 1, inputs)
    y = np.sin(x @ a / 3.0) + 0.5 * x[:, 0] * x[:, 1]
    with als.Surrogate(inputs, width, hidden, max_batch=1024, seed=1) as s:
        losses = s.fit(x, y, steps=400, lr=1e-3)
        pred = s(x).cpu().numpy()
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.02 * losses[0]
    resid = (y - pred).var() / y.var()
    assert resid < 0.02


def test_inference_in_chunks_is_row_independent():
    inputs = 40
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, (70000, inputs)).astype(np.float32)
    with als.Surrogate(seed=3) as s:
        full = s.forward_raw(x).cpu().numpy()
        part = s.forward_raw(x[65500:65700]).cpu().numpy()
    np.testing.assert_array_equal(full[65500:65700], part)


@pytest.mark.parametrize("inputs,hidden", [(40, 4), (64, 1), (7, 2), (33, 6)])
def test_whole_network_kernel_equals_the_per_layer_kernels(inputs, hidden):
    """The 256-wide network's inference runs as one kernel (activations kept
    on the SM); its outputs equal those of one kernel per layer bit for bit,
    for ragged row counts, a row count that crosses the 262,144-row chunk,
    and every depth.  The per-layer path is itself checked against the
    oracle above."""
    rng = np.random.default_rng(inputs * 10 + hidden)
    with als.Surrogate(inputs, 256, hidden, max_batch=1024, seed=hidden) as s:
        for rows in (1, 127, 255, 256, 257, 5000, 262144 + 300):
            x = torch.tensor(rng.uniform(0, 1, (rows, inputs)).astype(np.float32), device="cuda:0")
            fused = s.forward_raw(x).cpu().numpy()
            layered = s.forward_raw(x, per_layer=True).cpu().numpy()
            np.testing.assert_array_equal(fused, layered, err_msg="rows %d" % rows)


@pytest.mark.parametrize("hidden", [1, 6])
def test_whole_network_kernel_matches_oracle(hidden):
    inputs, rows = 40, 700
    rng = np.random.default_rng(hidden)
    x = rng.uniform(0, 1, (rows, inputs)).astype(np.float32)
    with als.Surrogate(inputs, 256, hidden, max_batch=1024, seed=13) as s:
        y = s.forward_raw(x).cpu().numpy().astype(np.float64)
        p = s.params()
    ref, _ = mo.forward(p, x, inputs, 256, hidden, bf16_path=True)
    scale = np.abs(ref).max() + 1e-3
    # the tolerances of test_forward_matches_oracle
    assert np.abs(y - ref).max() <= 1e-2 * scale, np.abs(y - ref).max()
    assert np.abs(y - ref).mean() <= 1e-3 * scale


def test_whole_network_inference_waits_for_the_callers_stream():
    """The inputs are written on the caller's stream after a bounded GPU
    sleep; the call (two chunks, the second one's inputs packed on the
    library's side stream) still sees them, on every chunk."""
    rows = 262144 + 4000
    gen = torch.Generator(device="cuda:0").manual_seed(5)
    src = torch.rand((rows, 40), device="cuda:0", generator=gen)
    with als.Surrogate(seed=9) as s:
        expect = s.forward_raw(src).cpu().numpy()
        x = torch.zeros_like(src)
        side = torch.cuda.Stream(device="cuda:0")
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            torch.cuda._sleep(50_000_000)      # about 25 ms of spinning on the GPU
            x.copy_(src)
            y = s.forward_raw(x)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(y.cpu().numpy(), expect)


def test_whole_network_kernel_wait_timeout_is_reported_and_the_handle_recovers():
    """Failure detection without a fault: with the layer completions of the
    whole-network kernel withheld, the epilogue's bounded waits run out, the
    roles drain their MMAs and copies, free tensor memory and return, and the
    call reports ALS_E_CUDA.  Afterwards the same handle gives the same
    outputs as before, bit for bit."""
    rng = np.random.default_rng(12)
    x = torch.tensor(rng.random((3000, 40), dtype=np.float32), device="cuda:0")
    with als.Surrogate(seed=5) as s:
        y0 = s.forward_raw(x).cpu().numpy()
        lib = als._lib.load()
        als._lib.check(lib.als_mlp_test_wait_timeout(s._h, 1024, 1))
        with pytest.raises(als._lib.AlsError) as err:
            s.forward_raw(x)
        assert err.value.code == -2 and "timed out" in str(err.value)
        als._lib.check(lib.als_mlp_test_wait_timeout(s._h, 0, 0))
        torch.cuda.synchronize()
        y1 = s.forward_raw(x).cpu().numpy()
    np.testing.assert_array_equal(y0, y1)


def test_device_uniform_draws_and_moments():
    with als.Surrogate(seed=3) as s:
        x = torch.empty(40 * 4096, dtype=torch.float32, device="cuda")
        from alsvinn_b200 import _lib
        _lib.check(s._lib.als_mlp_sample_uniform(x.data_ptr(), x.numel(), 7, 0))
        torch.cuda.synchronize()
        xs = x.cpu().numpy()
        assert xs.min() >= 0.0 and xs.max() < 1.0
        assert abs(xs.mean() - 0.5) < 5e-3
        m1, m2 = s.moments(1 << 18, seed=1)
        f = s(x.view(4096, 40)).double().cpu().numpy()
    assert abs(m1 - f.mean()) < 5 * f.std() / np.sqrt(4096)
    assert m2 >= m1 * m1


def _heldout_reduction(params, y, train, val, held, steps=2000):
    with als.Surrogate(seed=0) as s:
        s.fit(params[train], y[train], steps=steps, lr=1e-3,
              validation=(params[val], y[val]), check_every=50)
        f = s(params[held]).double().cpu().numpy()
        m1, m2 = s.moments(1 << 20, seed=2)
    yh = y[held]
    fc = f - f.mean()
    beta = np.dot(fc, yh - yh.mean()) / np.dot(fc, fc)
    return np.var(yh - beta * f) / np.var(yh), f, m1, m2


def test_control_variate_gain_on_early_time_samples():
    """Solver-generated samples (KH 256^2 to T = 0.2, FP32 members): a
    surrogate trained on 1024 of them (early stopping on 256) removes a
    large part of the observable's variance on 768 held-out samples, so the
    control-variate estimator needs proportionally fewer solver samples than
    plain MC for the same mean-square error."""
    params, y, info = als.uq.kh_observable_ensemble(256, 0, 2048, precision="fp32",
                                                    end_time=0.2)
    assert np.all(np.isfinite(y)) and y.std() > 0
    reduction, f, m1, m2 = _heldout_reduction(params, y, slice(0, 1024), slice(1024, 1280),
                                              slice(1280, 2048))
    assert reduction < 0.75, reduction
    # the estimator on the held-out samples agrees with plain MC within its error
    yh = y[1280:]
    mean_cv, var_cv, _, _ = als.uq.control_variate(yh, f, m1, m2)
    mean_pl, var_pl = als.uq.plain_mc(yh)
    assert abs(mean_cv - mean_pl) < 4 * np.sqrt(var_pl / yh.size)
    assert abs(var_cv - var_pl) < 0.5 * var_pl


def test_control_variate_gain_at_the_final_time():
    """The 4096-sample FP64 ensemble at T = 2 (committed fixture): trained on
    samples 0..1023, early-stopped on 1024..2047, evaluated on 2048..4095.  At
    T = 2 the observable is dominated by the chaotic roll-up, so the gain is
    small, but the control variate must still remove variance, never add it."""
    z = load_golden("uq_kh256_fp64_4096")
    y = np.asarray(z["y"], dtype=np.float64)
    params = als.uniform_draws(40, 0, y.size)
    reduction, _, _, _ = _heldout_reduction(params, y, slice(0, 1024), slice(1024, 2048),
                                            slice(2048, 4096))
    assert reduction < 0.95, reduction


def test_gemm_wait_timeout_is_reported_and_the_handle_recovers():
    """Failure detection without a fault: with the completion commits of
    the training GEMMs withheld, their mbarrier waits run out after a short
    poll limit, the kernels drain their MMAs, free tensor memory and return,
    and the call reports ALS_E_CUDA.  Afterwards the same handle computes the
    same gradients as before, bit for bit, and trains again."""
    rng = np.random.default_rng(11)
    x = torch.tensor(rng.random((300, 40), dtype=np.float32), device="cuda:0")
    t = torch.tensor(rng.standard_normal(300).astype(np.float32), device="cuda:0")
    with als.Surrogate(seed=5) as s:
        g0, l0 = s.gradients(x, t)
        g0 = g0.cpu().numpy()
        lib = als._lib.load()
        als._lib.check(lib.als_mlp_test_wait_timeout(s._h, 1024, 1))
        with pytest.raises(als._lib.AlsError) as err:
            s.gradients(x, t)
        assert err.value.code == -2 and "timed out" in str(err.value)
        with pytest.raises(als._lib.AlsError) as err:
            s.train_raw(x, t, 3)
        assert err.value.code == -2
        als._lib.check(lib.als_mlp_test_wait_timeout(s._h, 0, 0))
        torch.cuda.synchronize()
        # training above ran Adam on garbage gradients: restore the parameters
        s.init(5)
        g1, l1 = s.gradients(x, t)
        # gradients are reduced in a fixed order; the loss is summed with atomics
        assert np.array_equal(g1.cpu().numpy(), g0) and abs(l1 - l0) <= 1e-6 * abs(l0)
        loss = s.train_raw(x, t, 5)
        assert np.all(np.isfinite(loss)) and loss[-1] < loss[0]
