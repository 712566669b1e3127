"""The force-correction network (no reference counterpart): forward, gradients and
training through the C ABI against a PyTorch-CPU conv3d restatement that rounds to
bf16 at the same points (inputs, weights, hidden activations)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NN_TOL = 2e-2       # bf16 operands: relative to the largest entry
GRAD_TOL = 4e-2     # gradients also pass bf16 cotangents through the GEMMs


@pytest.fixture(scope="module")
def djb(cuda_device):
    import djb200
    return djb200


def _bf16(t):
    import torch
    return t.to(torch.bfloat16).to(torch.float32)


def _torch_net(net, params):
    """(weights, biases) as torch CPU tensors in conv3d layout, bf16-rounded weights."""
    import torch
    ws, bs = [], []
    for (woff, wshape, boff, op, ci, co) in net.layout():
        W = params[woff:woff + int(np.prod(wshape))].reshape(wshape)      # [tap][ci_pad][co_pad]
        w = np.transpose(W[:, :ci, :co], (2, 1, 0)).reshape(co, ci, 3, 3, 3)  # tap = kz*9 + ky*3 + kx
        ws.append(_bf16(torch.tensor(w, requires_grad=False)).requires_grad_(True))
        bs.append(torch.tensor(params[boff:boff + co], requires_grad=True))
    return ws, bs


def _torch_forward(ws, bs, x):
    import torch
    import torch.nn.functional as F
    a = _bf16(torch.tensor(x)[None])
    for l, (w, b) in enumerate(zip(ws, bs)):
        y = F.conv3d(F.pad(a, (1, 1, 1, 1, 1, 1), mode="circular"), w) + b[None, :, None, None, None]
        if l < len(ws) - 1:
            a = _bf16(torch.relu(y))
        else:
            return y[0]


def test_forward_and_gradients_vs_torch(djb):
    import torch
    from djb200.nn import ForceNet
    rng = np.random.default_rng(0)
    res = 12
    x = rng.standard_normal((4, res, res, res)).astype(np.float32)
    t = rng.standard_normal((3, res, res, res)).astype(np.float32)
    with ForceNet(layers=3, cin=4, hidden=16, cout=3, seed=7) as net:
        p = net.get_params()
        out = net.apply(x)
        loss = net.backward(x, t)
        g = net.grads()
    ws, bs = _torch_net(net, p)
    ref = _torch_forward(ws, bs, x)
    r = ref.detach().numpy()
    assert np.max(np.abs(out - r)) < NN_TOL * np.max(np.abs(r))
    L = torch.mean((ref - torch.tensor(t)) ** 2)
    L.backward()
    assert abs(loss - float(L)) < 1e-3 * float(L)
    for (woff, wshape, boff, op, ci, co), w, b in zip(net.layout(), ws, bs):
        gw = g[woff:woff + int(np.prod(wshape))].reshape(wshape)[:, :ci, :co]
        gw_ref = np.transpose(w.grad.numpy().reshape(co, ci, 27), (2, 1, 0))
        assert np.max(np.abs(gw - gw_ref)) < GRAD_TOL * np.max(np.abs(gw_ref))
        gb = g[boff:boff + co]
        assert np.max(np.abs(gb - b.grad.numpy())) < GRAD_TOL * np.max(np.abs(b.grad.numpy()))
        # the padding entries stay zero
        assert np.all(g[woff:woff + int(np.prod(wshape))].reshape(wshape)[:, ci:, :] == 0)


def test_adam_step_matches_torch_adam(djb):
    import torch
    from djb200.nn import ForceNet
    rng = np.random.default_rng(1)
    res = 10
    x = rng.standard_normal((4, res, res, res)).astype(np.float32)
    t = rng.standard_normal((3, res, res, res)).astype(np.float32)
    with ForceNet(layers=2, cin=4, hidden=8, cout=3, seed=3) as net:
        p0 = net.get_params()
        net.backward(x, t)
        g = net.grads()
        net.adam_step(1e-3)
        p1 = net.get_params()
    # Adam's first step from zero moments with these gradients
    q = torch.tensor(p0.copy(), requires_grad=True)
    opt = torch.optim.Adam([q], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    q.grad = torch.tensor(g)
    opt.step()
    live = g != 0
    assert np.max(np.abs(p1[live] - q.detach().numpy()[live])) < 1e-6
    assert np.all(p1[~live] == p0[~live])


def test_training_reduces_loss_on_mesh_fields(djb):
    """A few Adam steps on a force-correction pair (64³ particles, 32³ mesh vs 64³)."""
    from djb200.nn import ForceNet, force_correction_pair
    c = djb.Cosmology(Omega_c=0.261, Omega_b=0.049, h=0.677, n_s=0.965, sigma8=0.81)
    x, t = force_correction_pair(c, n=32, boxsize=100.0, res=32, seed=2)
    assert tuple(x.shape) == (4, 32, 32, 32) and tuple(t.shape) == (3, 32, 32, 32)
    scale = float(t.abs().max())
    t = (t / scale).contiguous()
    x = x.clone()
    x[1:] /= float(x[1:].abs().max())
    with ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=1) as net:
        l0 = net.train_step(x, t, lr=1e-3)
        for _ in range(40):
            l1 = net.train_step(x, t, lr=1e-3)
    assert l1 < 0.7 * l0


@pytest.mark.parametrize("res", [20, 35])
def test_tensor_core_convolution_matches_im2col_and_torch(djb, res):
    """The tcgen05 implicit-GEMM forward (partial 8 × 16 tiles when res is not a
    multiple of the tile, several z segments) against the im2col + cuBLAS path and the
    PyTorch restatement, for the 4-layer, 32-channel network."""
    from djb200.nn import ForceNet
    rng = np.random.default_rng(res)
    x = rng.standard_normal((4, res, res, res)).astype(np.float32)
    with ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=5) as net:
        p = net.get_params()
        out_tc = net.apply(x)
        net.set_conv("im2col")
        out_gemm = net.apply(x)
        net.set_conv("tensor")
        again = net.apply(x)
    assert np.array_equal(out_tc, again)
    scale = np.max(np.abs(out_gemm))
    assert np.max(np.abs(out_tc - out_gemm)) < 1e-2 * scale
    ws, bs = _torch_net(net, p)
    r = _torch_forward(ws, bs, x).detach().numpy()
    assert np.max(np.abs(out_tc - r)) < NN_TOL * np.max(np.abs(r))


@pytest.mark.parametrize("res", [20, 40])
def test_tensor_core_backward_matches_im2col(djb, res):
    """Weight, bias and data gradients on the tensor cores (data gradients with the
    flipped, transposed weights and the ReLU mask fused; weight gradients from four
    staged planes as one 128-row operand, three passes) against the im2col + cuBLAS
    backward; at 40³ interior planes arrive by bulk tensor copies."""
    from djb200.nn import ForceNet
    rng = np.random.default_rng(res)
    x = rng.standard_normal((4, res, res, res)).astype(np.float32)
    t = rng.standard_normal((3, res, res, res)).astype(np.float32)
    with ForceNet(layers=4, cin=4, hidden=32, cout=3, seed=9) as net:
        l_tc = net.backward(x, t)
        g_tc = net.grads()
        net.set_conv("im2col")
        l_ref = net.backward(x, t)
        g_ref = net.grads()
    assert abs(l_tc - l_ref) < 1e-3 * l_ref
    for (woff, wshape, boff, op, ci, co) in net.layout():
        n = int(np.prod(wshape))
        gw, gw_ref = g_tc[woff:woff + n], g_ref[woff:woff + n]
        assert np.max(np.abs(gw - gw_ref)) < 2e-2 * np.max(np.abs(gw_ref))
        gb, gb_ref = g_tc[boff:boff + op], g_ref[boff:boff + op]
        assert np.max(np.abs(gb - gb_ref)) < 2e-2 * np.max(np.abs(gb_ref))
