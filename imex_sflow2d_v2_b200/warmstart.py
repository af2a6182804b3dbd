"""Training the Newton warm-start network on pairs harvested from the solver.

The pairs live in the context's device buffers (imex_gpu_harvest_data); torch
views them without a copy, computes the normalisation (mean and standard
deviation per input and target) and the normalised training set, and the
library's own kernels train the network (imex_mlp_train)."""
import ctypes as C

import numpy as np


class _DevArray:
    """__cuda_array_interface__ view of a float32 device buffer."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False),
                                         "version": 3}


def harvested(solver):
    """The harvested pairs as torch float32 tensors (x: (n,12), y: (n,2))."""
    import torch
    xp, yp, n = solver.harvest_data()
    if n == 0:
        return None, None
    x = torch.as_tensor(_DevArray(xp, (n, 12)), device="cuda")
    y = torch.as_tensor(_DevArray(yp, (n, 2)), device="cuda")
    return x, y


def train(net, solver, epochs=4, batch=4096, lr=2e-3, seed=11):
    """Normalise the harvested pairs, train `net` on them, set its
    normalisation.  Returns (pairs, per-epoch mean squared error in
    normalised units)."""
    import torch
    x, y = harvested(solver)
    if x is None:
        raise RuntimeError("no harvested training pairs")
    ok = torch.isfinite(x).all(1) & torch.isfinite(y).all(1)
    x, y = x[ok], y[ok]
    xm, xs = x.double().mean(0), x.double().std(0)
    ym, ys = y.double().mean(0), y.double().std(0)
    xs = torch.where(xs > 1e-12, xs, torch.ones_like(xs))
    ys = torch.where(ys > 1e-30, ys, torch.ones_like(ys))
    xn = ((x.double() - xm) / xs).float().contiguous()
    yn = ((y.double() - ym) / ys).float().contiguous()
    net.set_norm(xm.cpu().numpy(), xs.cpu().numpy(), ym.cpu().numpy(), ys.cpu().numpy())
    losses = net.train(C.c_void_p(xn.data_ptr()), C.c_void_p(yn.data_ptr()), xn.shape[0],
                       epochs=epochs, batch=batch, lr=lr, seed=seed)
    torch.cuda.synchronize()
    return int(xn.shape[0]), np.asarray(losses)
