"""Cost model of the gapped stage: the NumPy gradient oracle against finite
differences (CPU), the CUDA training kernels' gradients and the BF16
inference against the oracle (GPU)."""
import numpy as np
import pytest

import cost_model_ref as R


def _data(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.random((n, R.FEAT)).astype(np.float32) * 2
    Y = (4 + 3 * X[:, 0] + 2 * np.sin(3 * X[:, 1]) + X[:, 4] * X[:, 6]).astype(np.float32)
    return X, Y


def _params(seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(R.PARAMS) * 0.3).astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    X, Y = _data(1, 64)
    p = _params(2).astype(np.float64)
    _, g = R.loss_and_grad(p, X, Y)
    rng = np.random.default_rng(3)
    for i in rng.choice(R.PARAMS, 60, replace=False):
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (R.loss_and_grad(pp, X, Y)[0] - R.loss_and_grad(pm, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), i


def test_param_layout_matches_library():
    from gzb import native as N
    assert N.cost_param_count() == R.PARAMS


@pytest.mark.gpu
def test_gpu_gradients_match_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes as C
    from gzb import native as N
    for n in (1, 100, 777):
        X, Y = _data(10 + n, n)
        p = _params(20 + n)
        dp, dx, dy = (torch.from_numpy(a.copy()).cuda() for a in (p, X.reshape(-1), Y))
        dg = torch.zeros(R.PARAMS, dtype=torch.float32, device="cuda")
        dl = torch.zeros(1, dtype=torch.float32, device="cuda")
        N.check(N.lib().gzb_cost_model_gradients(
            C.c_void_p(dp.data_ptr()), C.c_void_p(dx.data_ptr()), C.c_void_p(dy.data_ptr()), n,
            C.c_void_p(dg.data_ptr()), C.c_void_p(dl.data_ptr()), None))
        loss, g = R.loss_and_grad(p, X, Y)
        got = dg.cpu().numpy()
        assert np.allclose(got, g, rtol=1e-4, atol=1e-5 * max(1.0, np.abs(g).max()))
        assert abs(float(dl.cpu()[0]) - loss) <= 1e-4 * max(1.0, loss)


@pytest.mark.gpu
def test_gpu_bf16_inference_close_to_fp32_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes as C
    from gzb import native as N
    X, Y = _data(5, 5000)
    p = _params(6)
    dp, dx = (torch.from_numpy(a.copy()).cuda() for a in (p, X.reshape(-1)))
    out = torch.zeros(len(X), dtype=torch.float32, device="cuda")
    N.check(N.lib().gzb_cost_model_predict(C.c_void_p(dp.data_ptr()), C.c_void_p(dx.data_ptr()),
                                           len(X), C.c_void_p(out.data_ptr()), None))
    ref, _ = R.forward(p, X)
    got = out.cpu().numpy()
    # bf16 keeps 8 significant bits: compare relative to the output scale
    assert np.abs(got - ref).max() <= 0.05 * max(1.0, np.abs(ref).max())


@pytest.mark.gpu
def test_gpu_training_reduces_loss():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ctypes as C
    from gzb import native as N
    X, Y = _data(7, 20000)
    p0 = N.cost_model_init(11)
    l0, _ = R.loss_and_grad(p0, X, Y)
    dx, dy = (torch.from_numpy(a.copy()).cuda() for a in (X.reshape(-1), Y))
    p = p0.copy()
    loss = C.c_float()
    N.check(N.lib().gzb_cost_model_train(C.c_void_p(dx.data_ptr()), C.c_void_p(dy.data_ptr()),
                                         len(X), N.hptr(p), 8, 1024, 3e-3, 5, C.byref(loss), None))
    l1, _ = R.loss_and_grad(p, X, Y)
    assert l1 < 0.1 * l0
    assert abs(loss.value - l1) <= 1e-3 * max(1.0, l1)
