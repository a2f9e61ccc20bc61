"""FP64 reference of the control-variate MLP -- TEST INFRASTRUCTURE ONLY.

16 -> 64 -> 64 -> 1 with SiLU, parameters packed as
W1[64][16] b1[64] W2[64][64] b2[64] w3[64] b3 (5313 values), loss
sum_r wt_r (f(x_r) - y_r)^2 * inv_wsum.  Used to check the device forward
and the device gradients (BF16 operands, FP32 accumulation) of
engineer-thesis_b200/csrc/cv.cu.
"""
import numpy as np

NIN, NH = 16, 64
O_W1, O_B1 = 0, NH * NIN
O_W2 = O_B1 + NH
O_B2 = O_W2 + NH * NH
O_W3 = O_B2 + NH
O_B3 = O_W3 + NH
NPARAM = O_B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[O_W1:O_B1].reshape(NH, NIN), p[O_B1:O_W2], p[O_W2:O_B2].reshape(NH, NH), p[O_B2:O_W3],
            p[O_W3:O_B3], p[O_B3])


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, round_operands=True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    if round_operands:  # the device multiplies BF16 copies of x, W1, W2
        x, W1, W2 = bf16(x), bf16(W1), bf16(W2)
    z1 = x @ W1.T + b1
    h1 = silu(z1)
    z2 = (bf16(h1) if round_operands else h1) @ W2.T + b2
    h2 = silu(z2)
    return h2 @ w3 + b3, (x, W1, W2, z1, h1, z2, h2)


def loss_grad(p, x, y, wt, inv_wsum, round_operands=True):
    out, (x, W1, W2, z1, h1, z2, h2) = forward(p, x, round_operands)
    _, _, _, _, w3, _ = unpack(p)
    e = out - y
    loss = float(np.sum(wt * e * e) * inv_wsum)
    d = 2.0 * wt * e * inv_wsum
    g = np.zeros(NPARAM)
    g[O_B3] = d.sum()
    g[O_W3:O_B3] = d @ h2
    dz2 = np.outer(d, w3) * dsilu(z2)
    g[O_B2:O_W3] = dz2.sum(0)
    g[O_W2:O_B2] = (dz2.T @ h1).ravel()
    dz1 = (dz2 @ W2) * dsilu(z1)
    g[O_B1:O_W2] = dz1.sum(0)
    g[O_W1:O_B1] = (dz1.T @ x).ravel()
    return loss, g
