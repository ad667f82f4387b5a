"""Differentiable CP loss (torch.autograd.Function over the MTTKRP kernels):
value vs the explicit reconstruction, gradient vs FP64 central finite
differences and vs the reference's gradient form F_n G_{-n} - M_n
(ntf/ntfnes.hpp:138-147) evaluated with the CPU oracle's MTTKRP."""
import numpy as np
import pytest

from helpers import cp_tensor, rel

pytestmark = pytest.mark.gpu


def _setup(prec, dims=(64, 64, 64), k=8, seed=31):
    import torch
    from planc_b200.autograd import CPLoss
    X, _ = cp_tensor(dims, k, noise=0.05, seed=seed)
    rng = np.random.default_rng(seed + 1)
    F = [rng.random((d, k)) for d in dims]
    lossf = CPLoss(X if prec == "fp64" else X.astype(np.float32), rank=k, precision=prec)
    Ft = [torch.tensor(f, device="cuda", dtype=torch.float64, requires_grad=True) for f in F]
    return X, F, lossf, Ft


def test_cp_loss_value_and_reference_gradient(gpu, oracle_lib):
    X, F, lossf, Ft = _setup("fp64")
    loss = lossf(*Ft)
    loss.backward()
    model = np.einsum("az,bz,cz->abc", *F)
    ref_loss = 0.5 * np.sum((X - model) ** 2)
    assert abs(loss.item() - ref_loss) / ref_loss < 1e-10
    for n in range(3):
        M = oracle_lib.mttkrp_direct(X, F, n)
        G = oracle_lib.gram_loo(F, n)
        ref_grad = F[n] @ G - M
        assert rel(Ft[n].grad.cpu().numpy(), ref_grad) < 1e-10
    lossf.close()


def test_cp_loss_gradient_finite_differences(gpu):
    import torch
    X, F, lossf, Ft = _setup("fp64", seed=33)
    loss = lossf(*Ft)
    loss.backward()
    rng = np.random.default_rng(7)
    h = 1e-5
    for n in range(3):
        E = torch.tensor(rng.standard_normal(F[n].shape), device="cuda", dtype=torch.float64)
        with torch.no_grad():
            plus = [f.detach().clone() for f in Ft]
            minus = [f.detach().clone() for f in Ft]
            plus[n] += h * E
            minus[n] -= h * E
            fd = (lossf(*plus).item() - lossf(*minus).item()) / (2 * h)
        an = float((Ft[n].grad * E).sum())
        assert abs(fd - an) / abs(an) < 1e-6, (n, fd, an)
    lossf.close()


@pytest.mark.parametrize("prec", ["bf16", "bf16x2"])
def test_cp_loss_mixed_precision_gradient(gpu, prec):
    X, F, lossf, Ft = _setup("fp64", seed=35)
    loss64 = lossf(*Ft)
    loss64.backward()
    g64 = [f.grad.clone() for f in Ft]
    lossf.close()
    _, _, lossf2, Ft2 = _setup(prec, seed=35)
    loss = lossf2(*Ft2)
    loss.backward()
    bound = 4e-3 if prec == "bf16" else 2e-5
    for a, b in zip(Ft2, g64):
        assert rel(a.grad.cpu().numpy(), b.cpu().numpy()) < bound
    lossf2.close()


def test_projected_gradient_descent_decreases_loss(gpu):
    # block-coordinate projected gradient steps, step 1/L_n with L_n the
    # largest eigenvalue of the leave-one-out Gram product: every step is a
    # descent step for the block it moves
    import torch
    X, F, lossf, Ft = _setup("fp64", dims=(48, 40, 32), k=6, seed=37)
    losses = []
    for it in range(10):
        for n in range(3):
            for f in Ft:
                f.grad = None
            loss = lossf(*Ft)
            loss.backward()
            losses.append(loss.item())
            with torch.no_grad():
                others = [g for m, g in enumerate(Ft) if m != n]
                Lc = float(torch.linalg.matrix_norm((others[0].T @ others[0]) * (others[1].T @ others[1]), 2))
                Ft[n].sub_(Ft[n].grad / Lc).clamp_(min=0.0)
    assert all(b <= a * (1 + 1e-6) for a, b in zip(losses, losses[1:]))
    assert losses[-1] < 0.5 * losses[0]
    lossf.close()


@pytest.mark.parametrize("prec", ["fp64", "bf16x2"])
def test_cp_loss_4way_reference_gradient(gpu, oracle_lib, prec):
    # 4-way: the backward's in-order reuse walks both branches of the tree
    import torch
    from planc_b200.autograd import CPLoss
    dims, k = (20, 16, 24, 12), 5
    X, _ = cp_tensor(dims, k, noise=0.05, seed=51)
    rng = np.random.default_rng(52)
    F = [rng.random((d, k)) for d in dims]
    lossf = CPLoss(X if prec == "fp64" else X.astype(np.float32), rank=k, precision=prec)
    Ft = [torch.tensor(f, device="cuda", dtype=torch.float64, requires_grad=True) for f in F]
    loss = lossf(*Ft)
    loss.backward()
    bound = 1e-10 if prec == "fp64" else 2e-5
    for n in range(4):
        M = oracle_lib.mttkrp_direct(X, F, n)
        G = oracle_lib.gram_loo(F, n)
        ref_grad = F[n] @ G - M
        assert rel(Ft[n].grad.cpu().numpy(), ref_grad) < bound, (n, rel(Ft[n].grad.cpu().numpy(), ref_grad))
    lossf.close()


@pytest.mark.parametrize("dims", [(40, 36, 28), (20, 16, 24, 12)])
def test_cp_loss_backward_after_second_forward(gpu, dims):
    # two forwards on one CPLoss, then the FIRST loss's backward: its gradient
    # must be built from its own factors, not from the tree state the second
    # forward left in the context (checked against torch autograd of the
    # dense FP64 reconstruction)
    import torch
    from planc_b200.autograd import CPLoss
    k = 5
    X, _ = cp_tensor(dims, k, noise=0.05, seed=61)
    rng = np.random.default_rng(62)
    F1 = [rng.random((d, k)) for d in dims]
    F2 = [rng.random((d, k)) for d in dims]
    lossf = CPLoss(X, rank=k, precision="fp64")
    A = [torch.tensor(f, device="cuda", dtype=torch.float64, requires_grad=True) for f in F1]
    B = [torch.tensor(f, device="cuda", dtype=torch.float64, requires_grad=True) for f in F2]
    loss_a = lossf(*A)
    loss_b = lossf(*B)
    loss_a.backward()
    loss_b.backward()
    Xt = torch.tensor(X, device="cuda", dtype=torch.float64)
    letters = "abcd"[:len(dims)]
    spec = ",".join(c + "z" for c in letters) + "->" + letters
    for got, F in ((A, F1), (B, F2)):
        R = [torch.tensor(f, device="cuda", dtype=torch.float64, requires_grad=True) for f in F]
        ref = 0.5 * ((Xt - torch.einsum(spec, *R)) ** 2).sum()
        ref.backward()
        for g, r in zip(got, R):
            assert rel(g.grad.cpu().numpy(), r.grad.cpu().numpy()) < 1e-10
    lossf.close()


def test_projected_accelerated_step_kernel(gpu):
    # the fused step against the same arithmetic in torch, with outputs in
    # place of inputs of the same factor
    import torch
    from planc_b200.autograd import projected_accelerated_step
    X, F, lossf, Ft = _setup("fp64", dims=(30, 20, 10), k=4, seed=41)
    rng = np.random.default_rng(42)
    Y = [torch.tensor(rng.random(f.shape), device="cuda", dtype=torch.float64) for f in F]
    Gr = [torch.tensor(rng.standard_normal(f.shape), device="cuda", dtype=torch.float64) for f in F]
    P = [torch.tensor(rng.random(f.shape), device="cuda", dtype=torch.float64) for f in F]
    eta, mom = 0.37, 0.61
    refF = [(y - eta * g).clamp(min=0.0) for y, g in zip(Y, Gr)]
    refY = [nf + mom * (nf - p) for nf, p in zip(refF, P)]
    Fn = [torch.empty_like(y) for y in Y]
    projected_accelerated_step(lossf, Y, Gr, P, eta, mom, Fn, Y)  # Ynew written over Y
    torch.cuda.synchronize()
    # the kernel forms y - eta g with one rounding (a fused multiply-add)
    for a, b in zip(Fn, refF):
        assert torch.allclose(a, b, rtol=0, atol=1e-15)
    for a, b in zip(Y, refY):
        assert torch.allclose(a, b, rtol=0, atol=1e-14)
    lossf.close()


@pytest.mark.parametrize("prec", ["fp64", "bf16"])
def test_cp_loss_captures_as_cuda_graph(gpu, prec):
    # forward + backward captured once on the loss's stream (static factor
    # inputs, static loss and gradients) replay the eager computation's bits
    import torch
    X, F, lossf, Ft = _setup(prec, dims=(48, 40, 36), k=8, seed=51)
    s = torch.cuda.ExternalStream(lossf.ctx.stream, device="cuda")
    Ys = [f.detach().clone().requires_grad_(True) for f in Ft]
    eager = []
    with torch.cuda.stream(s):
        for step in range(3):
            for y in Ys:
                y.grad = None
            loss = lossf(*Ys)
            loss.backward()
            eager.append((loss.detach().clone(), [y.grad.clone() for y in Ys]))
            with torch.no_grad():
                for y in Ys:
                    y.mul_(0.9)
    torch.cuda.synchronize()
    with torch.no_grad():
        for y, f in zip(Ys, Ft):
            y.copy_(f.detach())
    for y in Ys:
        y.grad = None
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="relaxed"):
        static_loss = lossf(*Ys)
        static_loss.backward()
    grads = [y.grad for y in Ys]
    with torch.no_grad():
        for y, f in zip(Ys, Ft):
            y.copy_(f.detach())
    with torch.cuda.stream(s), torch.no_grad():
        for step in range(3):
            graph.replay()
            torch.cuda.synchronize()
            el, eg = eager[step]
            assert torch.equal(static_loss, el), step
            assert all(torch.equal(a, b) for a, b in zip(grads, eg)), step
            for y in Ys:
                y.mul_(0.9)
    del graph
    lossf.close()
