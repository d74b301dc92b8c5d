"""TEST INFRASTRUCTURE ONLY: a float64 restatement of the warm-start network
(aero_mlp_* in aerocfd_b200/csrc/aero_mlp.cu) for checking its tensor-core
forward pass and gradients.  It rounds to BF16 where the device does (inputs,
weights, activations, the backward signals fed to the GEMMs) and computes
everything else in float64; the device accumulates in FP32, so the two agree
to the BF16 rounding of values that sit next to a rounding boundary.

Parameter layout (as aero_mlp_get_params): per layer W [nout x nin] row-major
then b [nout]; input and output layers padded to 128."""
import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32).astype(np.float64)


def unpack(params, n_in_pad, width, depth, n_out_pad):
    layers, o = [], 0
    for l in range(depth + 1):
        nin = n_in_pad if l == 0 else width
        nout = n_out_pad if l == depth else width
        W = params[o:o + nin * nout].reshape(nout, nin).astype(np.float64)
        o += nin * nout
        b = params[o:o + nout].astype(np.float64)
        o += nout
        layers.append((W, b))
    return layers


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(layers, x, n_in_pad=128):
    h = np.zeros((x.shape[0], n_in_pad))
    h[:, :x.shape[1]] = x
    hs, zs = [bf16(h)], []
    for W, b in layers[:-1]:
        z = hs[-1] @ bf16(W).T + b.astype(np.float32).astype(np.float64)
        zs.append(z)
        hs.append(bf16(silu(z)))
    W, b = layers[-1]
    y = hs[-1] @ bf16(W).T + b
    return y, hs, zs


def loss_and_grads(layers, x, t):
    n, n_out = t.shape
    y, hs, zs = forward(layers, x)
    d = np.zeros_like(y)
    d[:, :n_out] = y[:, :n_out] - t
    loss = np.sum(d ** 2) / (n * n_out)
    dyf = 2.0 * d / (n * n_out)
    dy = bf16(dyf)
    grads = [None] * len(layers)
    W, _ = layers[-1]
    grads[-1] = (dy.T @ hs[-1], dyf.sum(axis=0))
    dh = dy @ bf16(W)
    for l in range(len(layers) - 2, -1, -1):
        z = zs[l]
        s = 1.0 / (1.0 + np.exp(-z))
        dzf = dh * (s * (1.0 + z * (1.0 - s)))
        dz = bf16(dzf)
        grads[l] = (dz.T @ hs[l], dzf.sum(axis=0))
        if l > 0:
            dh = dz @ bf16(layers[l][0])
    return loss, grads, y
