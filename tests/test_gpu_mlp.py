"""The learned pruner's GPU kernels through the C ABI against the numpy
oracle (oracle/mlp_oracle.py): the FP32 forward pass, the BF16 tensor-core
inference, the gradients of the training kernel and one Adam step, and a
short training run that must lower the loss."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FWD_RTOL, FWD_ATOL = 1e-4, 1e-4          # FP32 forward vs FP64 oracle
GRAD_RTOL = 2e-3                          # FP32 gradients vs FP64 oracle, relative to the largest entry
BF16_ATOL, BF16_RTOL = 0.08, 0.05         # BF16 weights/activations, FP32 accumulation


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _case(n=777, seed=0):
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(seed)
    theta = mo.init(seed).astype(np.float32)
    theta[mo.NF * 64:mo.NF * 64 + 64] = rng.normal(0, 0.1, 64)        # non-zero biases
    x = rng.normal(size=(n, mo.NF)).astype(np.float32)
    y = (rng.uniform(size=(n, mo.NO)) < 0.25).astype(np.float32)
    return theta, x, y


def test_forward_fp32_matches_oracle():
    import torch
    from oracle import mlp_oracle as mo
    from tsr_b200 import core
    theta, x, _ = _case()
    out = torch.empty((x.shape[0], 2), device="cuda")
    xd, td = _dev(x), _dev(theta)      # keep the device copies alive until the kernel ran
    core._check(core.lib.tsr_mlp_forward(_p(xd), x.shape[0], _p(td), _p(out), _stream()))
    np.testing.assert_allclose(out.cpu().numpy(), mo.forward(theta, x), rtol=FWD_RTOL, atol=FWD_ATOL)


def test_bf16_inference_matches_oracle():
    import torch
    from oracle import mlp_oracle as mo
    from tsr_b200 import core
    theta, x, _ = _case(n=1000 + 13)            # not a multiple of the 16-row tile
    out = torch.full((x.shape[0], 2), float("nan"), device="cuda")
    xd, td = _dev(x), _dev(theta)
    core._check(core.lib.tsr_mlp_infer_bf16(_p(xd), x.shape[0], _p(td), _p(out), _stream()))
    z = out.cpu().numpy()
    ref = mo.forward(theta, x)
    assert np.isfinite(z).all()
    np.testing.assert_allclose(z, ref, rtol=BF16_RTOL, atol=BF16_ATOL)
    confident = np.abs(ref) > 0.5
    assert np.all(np.sign(z[confident]) == np.sign(ref[confident]))


def test_training_gradient_matches_oracle():
    import torch
    from oracle import mlp_oracle as mo
    from tsr_b200 import core
    theta, x, y = _case(n=300, seed=5)
    grads = torch.zeros(mo.NPARAM, device="cuda")
    loss = torch.zeros(1, device="cuda")
    xd, yd, td = _dev(x), _dev(y), _dev(theta)
    core._check(core.lib.tsr_mlp_train_batch(_p(xd), _p(yd), x.shape[0], _p(td), _p(grads),
                                             _p(loss), 3.0, 2.0, _stream()))
    l_ref, g_ref = mo.loss_and_grad(theta, x, y, (3.0, 2.0))
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * abs(l_ref)
    g = grads.cpu().numpy()
    assert np.max(np.abs(g - g_ref)) <= GRAD_RTOL * np.max(np.abs(g_ref))


def test_adam_step_matches_reference():
    import torch
    from tsr_b200 import core
    rng = np.random.default_rng(2)
    n = 4994
    p0, g = rng.normal(size=n).astype(np.float32), rng.normal(size=n).astype(np.float32)
    m0, v0 = rng.normal(size=n).astype(np.float32) * 0.1, rng.uniform(size=n).astype(np.float32) * 0.1
    p, m, v = _dev(p0), _dev(m0), _dev(v0)
    step, lr, scale = 7, 1e-2, 0.5
    gd = _dev(g)
    core._check(core.lib.tsr_mlp_adam(_p(p), _p(gd), _p(m), _p(v), step, lr, scale, _stream()))
    gs = g.astype(np.float64) * scale
    m1 = 0.9 * m0 + 0.1 * gs
    v1 = 0.999 * v0 + 0.001 * gs * gs
    p1 = p0 - lr * (m1 / (1 - 0.9 ** step)) / (np.sqrt(v1 / (1 - 0.999 ** step)) + 1e-8)
    np.testing.assert_allclose(m.cpu().numpy(), m1, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(v.cpu().numpy(), v1, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(p.cpu().numpy(), p1, rtol=1e-5, atol=1e-6)


def test_short_training_lowers_the_loss():
    from oracle import mlp_oracle as mo
    from tsr_b200 import pruner
    rng = np.random.default_rng(11)
    x = rng.normal(size=(20000, mo.NF)).astype(np.float32)
    y = np.stack([x[:, 0] + 0.5 * x[:, 3] > 0.8, np.abs(x[:, 1]) < 0.3], 1).astype(np.float32)
    l0, _ = mo.loss_and_grad(pruner.he_init(0), x, y)
    theta = pruner.train(x, y, epochs=3, batch=2048, lr=3e-3, seed=0, pos_weight=(1.0, 1.0))
    l1, _ = mo.loss_and_grad(theta, x, y)
    assert l1 < 0.5 * l0, (l0, l1)
