"""The block-demand predictor's hand-written fp32 kernels against a float64
numpy backpropagation (oracle/mlp_oracle.py).

Tolerances: forward outputs within 1e-4 relative (fp32 accumulation of 80
products); gradients within 2e-3 relative in L2 norm over each tensor (fp32
sums over 32 CTAs x samples vs float64)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(t):
    import torch
    return torch.as_tensor(np.ascontiguousarray(t, dtype=np.float32)).cuda()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def random_case(n, seed=0):
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(seed)
    p = np.concatenate([rng.normal(0, 0.3, M.HID * M.IN), rng.normal(0, 0.1, M.HID),
                        rng.normal(0, 0.15, M.HID * M.HID), rng.normal(0, 0.1, M.HID),
                        rng.normal(0, 0.2, M.HID), [0.05]]).astype(np.float32)
    x = rng.normal(0, 1.0, (n, M.IN)).astype(np.float32)
    t = rng.normal(0, 1.0, n).astype(np.float32)
    return p, x, t


def test_forward_matches_float64(gw):
    import torch
    from oracle import mlp_oracle as M
    p, x, _ = random_case(300, 1)
    y = torch.zeros(300, dtype=torch.float32, device="cuda")
    assert gw.load().gw_mlp_forward(ptr(dev(p)), ptr(dev(x)), 300, ptr(y)) == 0
    ref, _ = M.forward(p.astype(np.float64), x)
    got = y.cpu().numpy().astype(np.float64)
    assert np.allclose(got, ref, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("n", [1, 37, 1280])
def test_gradients_match_float64(gw, n):
    import torch
    from oracle import mlp_oracle as M
    from gowalker_b200._abi import GW_MLP_GRAD_WS_FLOATS, GW_MLP_PARAMS
    p, x, t = random_case(n, 2 + n)
    grad = torch.zeros(GW_MLP_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    ws = torch.zeros(GW_MLP_GRAD_WS_FLOATS, dtype=torch.float32, device="cuda")
    assert gw.load().gw_mlp_grad(ptr(dev(p)), ptr(dev(x)), ptr(dev(t)), n, ptr(grad), ptr(loss), ptr(ws)) == 0
    ref_loss, ref_grad = M.loss_and_grad(p.astype(np.float64), x, t)
    g = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    o = 0
    for name, shape in M.SIZES:
        k = int(np.prod(shape))
        a, b = g[o:o + k], ref_grad[o:o + k]
        assert np.linalg.norm(a - b) <= 2e-3 * max(np.linalg.norm(b), 1e-6), name
        o += k
    # finite-difference spot check of the float64 reference itself
    eps = 1e-6
    for idx in (3, 1100, 5000, GW_MLP_PARAMS - 1):
        pp = p.astype(np.float64).copy()
        pp[idx] += eps
        lp, _ = M.loss_and_grad(pp, x, t)
        pp[idx] -= 2 * eps
        lm, _ = M.loss_and_grad(pp, x, t)
        assert abs((lp - lm) / (2 * eps) - ref_grad[idx]) < 1e-5 * max(1.0, abs(ref_grad[idx]))


def test_training_reduces_loss_and_is_deterministic(gw):
    import torch
    from gowalker_b200._abi import GW_MLP_GRAD_WS_FLOATS, GW_MLP_PARAMS
    rng = np.random.default_rng(5)
    n = 1280
    x = rng.normal(0, 1.0, (n, 16)).astype(np.float32)
    t = (np.log1p(np.abs(3 * x[:, 0])) + 0.5 * np.maximum(x[:, 1], 0)).astype(np.float32)
    finals = []
    for _ in range(2):
        p = torch.zeros(GW_MLP_PARAMS, dtype=torch.float32, device="cuda")
        ws = torch.zeros(GW_MLP_GRAD_WS_FLOATS + 3 * GW_MLP_PARAMS + 1, dtype=torch.float32, device="cuda")
        l0, l1 = ctypes.c_float(), ctypes.c_float()
        L = gw.load()
        assert L.gw_mlp_train(ptr(p), ptr(dev(x)), ptr(dev(t)), n, 1, 3e-3, 99, ptr(ws), ctypes.byref(l0)) == 0
        assert L.gw_mlp_train(ptr(p), ptr(dev(x)), ptr(dev(t)), n, 400, 3e-3, 99, ptr(ws), ctypes.byref(l1)) == 0
        assert l1.value < 0.2 * l0.value, (l0.value, l1.value)
        finals.append(p.cpu().numpy())
    assert np.array_equal(finals[0], finals[1])
