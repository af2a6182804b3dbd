"""FP64 restatement of the warm-start network's forward and backward passes
(test infrastructure).  It applies the same BF16 roundings as the tensor-core
path (weights, and every layer input), so the GPU and this reference differ
only by FP32 against FP64 accumulation."""
import numpy as np

IN, IN_P, HID, OUT, OUT_P = 12, 16, 64, 2, 8
OFF = {}
_o = 0
for name, size in (("W0", IN_P * HID), ("b0", HID), ("W1", HID * HID), ("b1", HID),
                   ("W2", HID * HID), ("b2", HID), ("W3", HID * OUT_P), ("b3", OUT_P)):
    OFF[name] = (_o, size)
    _o += size
NPARAM = _o


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float32)
    g = {}
    for name, (o, n) in OFF.items():
        v = p[o:o + n]
        if name == "W0":
            v = v.reshape(IN_P, HID)
        elif name in ("W1", "W2"):
            v = v.reshape(HID, HID)
        elif name == "W3":
            v = v.reshape(HID, OUT_P)
        g[name] = v
    return g


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_grad(p, x, y):
    P = unpack(p)
    n = x.shape[0]
    a0 = np.zeros((n, IN_P))
    a0[:, :IN] = bf16(x)
    W = [bf16(P["W0"]), bf16(P["W1"]), bf16(P["W2"]), bf16(P["W3"])]
    b = [P["b0"].astype(np.float64), P["b1"].astype(np.float64), P["b2"].astype(np.float64),
         P["b3"].astype(np.float64)]
    acts, zs = [a0], []
    a = a0
    for l in range(3):
        z = a @ W[l] + b[l]
        zs.append(z)
        a = bf16(silu(z).astype(np.float32))
        acts.append(a)
    yp = (a @ W[3] + b[3])[:, :OUT]
    r = yp - y
    count = n * OUT
    loss = float((r * r).sum() / count)
    dz = np.zeros((n, OUT_P))
    dz[:, :OUT] = 2.0 * r / count
    grads = {"W3": acts[3].T @ dz, "b3": dz.sum(0)}
    da = dz @ W[3].T
    for l in (2, 1, 0):
        dzl = da * silu_grad(zs[l])
        grads["W%d" % l] = acts[l].T @ dzl
        grads["b%d" % l] = dzl.sum(0)
        da = dzl @ W[l].T
    g = np.zeros(NPARAM)
    for name, (o, sz) in OFF.items():
        g[o:o + sz] = grads[name].ravel()
    return loss, g, yp
