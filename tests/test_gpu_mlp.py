"""The surrogate's MLP kernels (BF16 tensor-core GEMMs with FP32
accumulation, fused bias/GELU epilogues, backward pass, Adam).

Gradient check: loss and gradients of every ensemble member against a
float64 CPU reference of the same network that rounds to bf16 at the same
points as the kernels (GEMM inputs: normalised X, weights, activations,
output gradient, back-propagated dZ).  The GPU accumulates in FP32, so a
pre-activation can land on the other side of a bf16 rounding boundary;
tolerance: relative L2 error of each member's gradient vector 2e-2, loss
relative 1e-2.  Training: an ensemble fits a smooth 25 -> 3 map, the loss
falling by at least 20x, and its predictions agree with the targets.
"""
import numpy as np
import pytest
import torch

import mcml_gpu_b200.surrogate as sg


def bf(a):
    return torch.as_tensor(a, dtype=torch.float64).to(torch.bfloat16).to(torch.float64)


C_GELU = np.sqrt(2.0 / np.pi)


def gelu(z):
    """GELU, tanh form (the kernels' activation)."""
    return 0.5 * z * (1.0 + torch.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = torch.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3 * 0.044715 * z * z)


def cpu_reference(params, shapes, X, T, xm, xs, tm, ts):
    n, in_dim = X.shape
    in_pad = shapes[0][0]
    xn = np.zeros((n, in_pad))
    inv = np.where(xs > 0, 1.0 / np.where(xs > 0, xs, 1), 0.0)
    xn[:, :in_dim] = (X - xm) * inv
    x = bf(xn)
    Ws, bs, off = [], [], 0
    for fi, fo in shapes:
        Ws.append(torch.as_tensor(params[off:off + fi * fo].reshape(fi, fo), dtype=torch.float64))
        off += fi * fo
        bs.append(torch.as_tensor(params[off:off + fo], dtype=torch.float64))
        off += fo
    hs, zs = [x], []
    for l in range(len(shapes) - 1):
        z = hs[-1] @ bf(Ws[l]) + bs[l]
        zs.append(z)
        hs.append(bf(gelu(z)))
    y = hs[-1] @ bf(Ws[-1]) + bs[-1]
    t = (torch.as_tensor(T, dtype=torch.float64) - torch.as_tensor(tm)) / torch.as_tensor(ts)
    d = y - t
    loss = float((d * d).mean())
    dz = bf(2.0 * d / d.numel())
    grads = [None] * (2 * len(shapes))
    for l in range(len(shapes) - 1, -1, -1):
        grads[2 * l] = hs[l].T @ dz
        grads[2 * l + 1] = dz.sum(0)
        if l == 0:
            break
        dz = bf((dz @ bf(Ws[l]).T) * gelu_grad(zs[l - 1]))
    return loss, torch.cat([g.reshape(-1) for g in grads]).numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [192, 1024])  # 1024: the weight gradients split over the batch
def test_gradients_match_cpu_reference(n, gpu_available):
    rng = np.random.default_rng(0)
    in_dim, out_dim = 25, 3
    X = rng.normal(size=(n, in_dim)).astype(np.float32) * 2 + 1
    T = rng.normal(size=(n, out_dim)).astype(np.float32) * 3 - 2
    mlp = sg.MLP(in_dim, out_dim, hidden=64, depth=3, ensemble=2, seed=5)
    xm, xs = X.mean(0), X.std(0)
    xs[3] = 0.0  # a constant feature: normalised to 0
    tm, ts = T.mean(0), T.std(0)
    mlp.set_normalization(xm, xs, tm, ts)
    dev = torch.device("cuda", 0)
    loss, grads = mlp.gradients(torch.from_numpy(X).to(dev), torch.from_numpy(T).to(dev))
    for e in range(2):
        p = mlp.params(e)
        ref_loss, ref_g = cpu_reference(p, mlp.layer_shapes(), X, T, xm, xs, tm, ts)
        assert abs(loss[e] - ref_loss) <= 1e-2 * ref_loss
        rel = np.linalg.norm(grads[e] - ref_g) / np.linalg.norm(ref_g)
        assert rel < 2e-2, rel


@pytest.mark.gpu
def test_ensemble_learns_smooth_map(gpu_available):
    rng = np.random.default_rng(1)
    n = 32768
    X = rng.uniform(-1, 1, size=(n, 25)).astype(np.float32)
    W = rng.normal(size=(25, 3)) / 5
    T = (np.sin(X @ W) + 0.5 * (X[:, :3] ** 2)).astype(np.float32)
    mlp = sg.MLP(25, 3, hidden=128, depth=3, ensemble=4, seed=2)
    mlp.set_normalization(X.mean(0), X.std(0), T.mean(0), T.std(0))
    dev = torch.device("cuda", 0)
    Xt, Tt = torch.from_numpy(X).to(dev), torch.from_numpy(T).to(dev)
    first = mlp.train_epoch(Xt, Tt, batch=1024, lr=2e-3, seed=0)
    for e in range(1, 12):
        last = mlp.train_epoch(Xt, Tt, batch=1024, lr=2e-3, seed=e)
    assert np.all(last < first / 20), (first, last)
    mean, spread = mlp.predict(Xt[:4096])
    err = np.abs(mean.cpu().numpy() - T[:4096])
    assert float(np.mean(err)) < 0.05 * float(np.std(T)) * 4
    assert spread.shape == mean.shape and bool(torch.all(spread >= 0))


def cpu_forward(params, shapes, X, xm, xs, tm, ts):
    n, in_dim = X.shape
    xn = np.zeros((n, shapes[0][0]))
    inv = np.where(xs > 0, 1.0 / np.where(xs > 0, xs, 1), 0.0)
    xn[:, :in_dim] = (X - xm) * inv
    h = bf(xn)
    off = 0
    for l, (fi, fo) in enumerate(shapes):
        W = torch.as_tensor(params[off:off + fi * fo].reshape(fi, fo), dtype=torch.float64)
        off += fi * fo
        b = torch.as_tensor(params[off:off + fo], dtype=torch.float64)
        off += fo
        z = h @ bf(W) + b
        h = bf(gelu(z)) if l < len(shapes) - 1 else z
    return h.numpy() * ts + tm


@pytest.mark.gpu
@pytest.mark.parametrize("hidden,depth,n", [(256, 4, 300), (64, 3, 129), (128, 2, 1000),
                                            (64, 2, 70000)])  # 70000: several tiles per CTA
def test_tensor_core_forward_matches_cpu_reference(hidden, depth, n, gpu_available):
    """predict() runs the tcgen05 forward: ensemble mean and spread against
    a float64 CPU forward that rounds to bf16 where the kernel does (GEMM
    inputs).  Rows past a 128-row tile boundary and partial tiles included.
    Tolerance: 1e-2 of the targets' scale (a bf16 rounding of an
    activation can land on the other side of a boundary)."""
    rng = np.random.default_rng(7)
    X = rng.normal(size=(n, 25)).astype(np.float32)
    T = rng.normal(size=(n, 3)).astype(np.float32) * 2 + 1
    mlp = sg.MLP(25, 3, hidden=hidden, depth=depth, ensemble=2, seed=3)
    xm, xs, tm, ts = X.mean(0), X.std(0), T.mean(0), T.std(0)
    mlp.set_normalization(xm, xs, tm, ts)
    dev = torch.device("cuda", 0)
    mean, spread = mlp.predict(torch.from_numpy(X).to(dev))
    ys = np.stack([cpu_forward(mlp.params(e), mlp.layer_shapes(), X, xm, xs, tm, ts)
                   for e in range(2)])
    scale = float(np.abs(ys).mean())
    assert np.max(np.abs(mean.cpu().numpy() - ys.mean(0))) < 1e-2 * scale
    assert np.max(np.abs(spread.cpu().numpy() - ys.std(0))) < 1e-2 * scale


@pytest.mark.gpu
def test_tensor_arguments_are_checked(gpu_available):
    """Wrongly typed, strided or shaped inputs are rejected before any launch."""
    mlp = sg.MLP(25, 3, hidden=64, depth=3, ensemble=2, seed=1)
    dev = torch.device("cuda", 0)
    X = torch.zeros((64, 25), dtype=torch.float32, device=dev)
    T = torch.zeros((64, 3), dtype=torch.float32, device=dev)
    with pytest.raises(ValueError, match="float32"):
        mlp.predict(X.double())
    with pytest.raises(ValueError, match="contiguous"):
        mlp.predict(torch.zeros((25, 64), device=dev).t())
    with pytest.raises(ValueError, match="shape"):
        mlp.predict(X[:, :24].contiguous())
    with pytest.raises(ValueError, match="shape"):
        mlp.train_epoch(X, T[:32], batch=32)
    mean, spread = mlp.predict(X)  # the checked path still runs
    assert mean.shape == (64, 3) and spread.shape == (64, 3)


@pytest.mark.gpu
def test_pipeline_wait_timeout_is_reported_and_drained(gpu_available, monkeypatch):
    """Every wait of the tensor-core kernel is bounded.  With the bound cut
    to one poll (MCML_MLP_WAIT_POLLS, read when a network is created) the
    waits run out on purpose: predict() must return MCML_E_BUDGET after the
    kernel drained what it had issued (bit 1 of the status word, a failed
    drain, must stay clear), and the context must stay usable -- a network
    created afterwards with the normal bound predicts what a fresh one does."""
    from mcml_gpu_b200 import MCMLError
    rng = np.random.default_rng(11)
    n = 65536
    X = torch.from_numpy(rng.normal(size=(n, 25)).astype(np.float32)).cuda()
    monkeypatch.setenv("MCML_MLP_WAIT_POLLS", "1")
    tiny = sg.MLP(25, 3, hidden=256, depth=4, ensemble=2, seed=5)
    monkeypatch.delenv("MCML_MLP_WAIT_POLLS")
    with pytest.raises(MCMLError) as err:
        tiny.predict(X)
    assert err.value.status == -8  # MCML_E_BUDGET
    assert "drained" in err.value.message, err.value.message
    tiny.close()
    a = sg.MLP(25, 3, hidden=256, depth=4, ensemble=2, seed=5)
    b = sg.MLP(25, 3, hidden=256, depth=4, ensemble=2, seed=5)
    ma, sa = a.predict(X)
    mb, sb = b.predict(X)
    assert torch.equal(ma, mb) and torch.equal(sa, sb)
    assert bool(torch.isfinite(ma).all())


@pytest.mark.gpu
@pytest.mark.parametrize("hidden,depth,n", [(256, 4, 3000), (64, 3, 1000), (128, 2, 70000),
                                            (256, 1, 5000),   # depth 1: the output folded into layer 0
                                            (192, 2, 9000)])  # six 32-column chunks over four warps
def test_fused_forward_agrees_with_layer_by_layer(hidden, depth, n, gpu_available, monkeypatch):
    """With a hidden width that is a multiple of 64 and MCML_MLP_FUSED=1,
    predict() runs every layer of every member in one launch (the fused
    kernel, activations kept in each CTA's L2-resident scratch, the output
    layer folded into the last hidden layer's epilogue); without it, one
    launch per layer.  Both round to BF16 at the same points and issue the
    same tensor-core MMAs for the hidden layers; the output layer's FP32 sums
    are added in another order, so the two agree to a few units in the last
    place of the output scale -- also for a last batch of rows that is not a
    whole 1024-row batch."""
    rng = np.random.default_rng(13)
    X = torch.from_numpy(rng.normal(size=(n, 25)).astype(np.float32)).cuda()
    mlp = sg.MLP(25, 3, hidden=hidden, depth=depth, ensemble=4, seed=21)
    mlp.set_normalization(np.zeros(25), np.ones(25), np.zeros(3), np.ones(3))
    monkeypatch.setenv("MCML_MLP_FUSED", "1")
    fm, fs = mlp.predict(X)
    monkeypatch.setenv("MCML_MLP_FUSED", "0")
    lm, ls = mlp.predict(X)
    # both against the float64 CPU forward first, so a failure says which path is off
    Xn = X.cpu().numpy()
    z = np.zeros(25)
    ys = np.stack([cpu_forward(mlp.params(e), mlp.layer_shapes(), Xn, z, np.ones(25),
                               np.zeros(3), np.ones(3)) for e in range(4)])
    scale = float(np.abs(ys).mean())
    err_f = float(np.max(np.abs(fm.cpu().numpy() - ys.mean(0))))
    err_l = float(np.max(np.abs(lm.cpu().numpy() - ys.mean(0))))
    assert err_f < 1e-2 * scale and err_l < 1e-2 * scale, (err_f, err_l, scale)
    assert float((fm - lm).abs().max()) <= 1e-5 * scale, float((fm - lm).abs().max())
    assert float((fs - ls).abs().max()) <= 1e-4 * scale, float((fs - ls).abs().max())
