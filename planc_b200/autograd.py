"""Differentiable CP reconstruction loss on the B200 kernels.

    loss(F_0..F_{N-1}) = 1/2 ||X - [[F_0, ..., F_{N-1}]]||^2
                       = 1/2 ||X||^2 - <M_0, F_0> + 1/2 sum(*_n F_n^T F_n)

with M_n the mode-n MTTKRP. The gradient is the reference's NTF gradient form
(ntf/ntfnes.hpp:138-147, G_{-n} H^T - M^T in its k x I layout):

    d loss / d F_n = F_n (*_{m != n} F_m^T F_m) - M_n

The forward pass runs the mode-0 MTTKRP on the tensor-core (or FP64) kernel
of a planc_b200.Context and one fused launch for every factor's Gram and the
loss value; the hand-written backward runs the remaining modes' MTTKRPs on
the same kernels (the modes after 0 reuse the dimension tree's partial
contractions in order, starting from the forward pass's mode 0) and one fused
launch for every mode's gradient, so one forward + backward reads X twice. The context's tree epoch is recorded by
the forward; when anything else has run an MTTKRP on the context since (a
second forward before this backward, a direct call), the backward recomputes
mode 1 from the tensor instead of reusing another call's intermediates. Factors are float64 CUDA tensors of
shape (I_n, k), contiguous (row-major, the library's factor layout).
"""
import torch

from . import Context


class _CPLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, handle, *factors):
        factors = [f.contiguous() for f in factors]
        dev = factors[0].device
        k = factors[0].shape[1]
        stream = torch.cuda.ExternalStream(handle.stream, device=dev)
        M0 = torch.empty_like(factors[0])
        G = torch.empty(len(factors), k, k, dtype=torch.float64, device=dev)
        loss = torch.empty((), dtype=torch.float64, device=dev)
        ptrs = [f.data_ptr() for f in factors]
        stream.wait_stream(torch.cuda.current_stream(dev))
        handle.mttkrp_device(0, ptrs, M0.data_ptr(), dimtree=True, reuse=False)
        ctx.tree_epoch = handle.tree_epoch
        # Grams of every factor and 1/2||X||^2 - <M_0, F_0> + 1/2 sum(*_n G_n)
        handle.cp_loss_device(ptrs, M0.data_ptr(), G.data_ptr(), loss.data_ptr())
        torch.cuda.current_stream(dev).wait_stream(stream)
        ctx.handle = handle
        ctx.save_for_backward(M0, G, *factors)
        return loss

    @staticmethod
    def backward(ctx, g):
        M0, G, *factors = ctx.saved_tensors
        handle = ctx.handle
        dev = factors[0].device
        stream = torch.cuda.ExternalStream(handle.stream, device=dev)
        ptrs = [f.data_ptr() for f in factors]
        N = len(factors)
        Ms = [M0] + [torch.empty_like(factors[n]) for n in range(1, N)]
        grads = [torch.empty_like(f) for f in factors]
        gs = g.detach().to(device=dev, dtype=torch.float64).contiguous()
        stream.wait_stream(torch.cuda.current_stream(dev))
        # the tree holds this forward's mode-0 intermediates only if no other
        # MTTKRP ran on the context since
        fresh = handle.tree_epoch == ctx.tree_epoch
        for n in range(1, N):
            # in-order sweep with unchanged factors: every mode reuses the tree
            # state left by the previous one
            handle.mttkrp_device(n, ptrs, Ms[n].data_ptr(), dimtree=True,
                                 reuse=(n > 1) or fresh)
        # every mode's gradient g (F_n (*_{m != n} G_m) - M_n) in one launch
        handle.cp_grads_device(ptrs, G.data_ptr(), [m.data_ptr() for m in Ms], gs.data_ptr(),
                               [x.data_ptr() for x in grads])
        torch.cuda.current_stream(dev).wait_stream(stream)
        return (None, *grads)


def projected_accelerated_step(loss_fn, Y, grads, Fprev, eta, mom, Fnew, Ynew):
    """One projected accelerated gradient step on every factor, in one launch
    on the loss's context: Fnew = max(Y - eta grad, 0), Ynew = Fnew + mom
    (Fnew - Fprev). Lists of float64 CUDA tensors of the factors' shapes
    (outputs may be the inputs of the same factor)."""
    handle = loss_fn.ctx
    dev = Y[0].device
    stream = torch.cuda.ExternalStream(handle.stream, device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    handle.cp_step_device([t.data_ptr() for t in Y], [t.data_ptr() for t in grads],
                          [t.data_ptr() for t in Fprev], eta, mom, [t.data_ptr() for t in Fnew],
                          [t.data_ptr() for t in Ynew])
    torch.cuda.current_stream(dev).wait_stream(stream)


class CPLoss:
    """Holds the tensor on the device; call with the factor leaves.

        loss_fn = CPLoss(X_device_ptr_or_array, dims, rank, precision="bf16")
        loss = loss_fn(A, B, C); loss.backward()
    """

    def __init__(self, X, dims=None, rank=None, precision="fp64", device=0, dtype="f32"):
        import numpy as np
        self.ctx = Context(device, precision)
        if isinstance(X, torch.Tensor):
            X = X.contiguous()
            dims = tuple(dims)
            self.ctx.set_tensor(X.data_ptr(), dims=dims, dtype="f32" if X.dtype == torch.float32 else "f64")
        else:
            self.ctx.set_tensor(X)
            dims = X.shape
        self.dims = tuple(int(d) for d in dims)
        self.rank = rank
        # factors of the right rank give the context its buffers; their values are unused
        self.ctx.set_factors([np.ones((d, rank)) for d in self.dims])
        self.ctx._norm2 = self.ctx.tensor_norm2()

    def __call__(self, *factors):
        for f, d in zip(factors, self.dims):
            if f.dtype != torch.float64 or not f.is_cuda or tuple(f.shape) != (d, self.rank):
                raise ValueError("factors must be float64 CUDA tensors of shape (I_n, rank)")
        return _CPLoss.apply(self.ctx, *factors)

    def close(self):
        self.ctx.close()
