"""NumPy reference of the learned-guess network (test infrastructure only).

Only tests/ use this module, as the checker of the device training kernels:
the same network (14 -> 64 -> 64 -> 64 -> 4, ReLU), the same parameter
layout, and the same BF16 rounding points (weights, normalised inputs,
hidden activations, the output delta and the hidden deltas) with FP32
arithmetic in between.  The device kernels accumulate in a different order
(tensor-core fragments), so agreement is to FP32 rounding plus the
occasional BF16 rounding flip, not bit for bit.
"""
import numpy as np

NIN, NH, NOUT = 14, 64, 4
OFF_W1 = 36
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH * NH
OFF_W4 = OFF_B3 + NH
OFF_B4 = OFF_W4 + NOUT * NH
SIZE = OFF_B4 + NOUT


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(P):
    P = np.asarray(P, dtype=np.float32)
    return {
        "in_mean": P[0:NIN], "in_std": P[NIN:2 * NIN], "out_mean": P[2 * NIN:2 * NIN + NOUT],
        "out_std": P[2 * NIN + NOUT:2 * NIN + 2 * NOUT],
        "W1": P[OFF_W1:OFF_B1].reshape(NH, NIN), "b1": P[OFF_B1:OFF_W2],
        "W2": P[OFF_W2:OFF_B2].reshape(NH, NH), "b2": P[OFF_B2:OFF_W3],
        "W3": P[OFF_W3:OFF_B3].reshape(NH, NH), "b3": P[OFF_B3:OFF_W4],
        "W4": P[OFF_W4:OFF_B4].reshape(NOUT, NH), "b4": P[OFF_B4:SIZE],
    }


def loss_and_grad(P, samples):
    """Loss and gradient (SIZE floats, zeros for the statistics) of one
    batch of samples [n, 22] (features 0..13, targets 14..17)."""
    p = unpack(P)
    f32 = np.float32
    n = len(samples)
    x = bf16((samples[:, :NIN].astype(f32) - p["in_mean"]) / p["in_std"])
    W1, W2, W3, W4 = (bf16(p[k]) for k in ("W1", "W2", "W3", "W4"))
    h1 = bf16(np.maximum(x @ W1.T + p["b1"], 0))
    h2 = bf16(np.maximum(h1 @ W2.T + p["b2"], 0))
    h3 = bf16(np.maximum(h2 @ W3.T + p["b3"], 0))
    y = h3 @ W4.T + p["b4"]
    t = (samples[:, 14:18].astype(f32) - p["out_mean"]) / p["out_std"]
    e = y - t
    loss = float(np.mean(e.astype(np.float64) ** 2))
    dy = bf16(f32(2.0 / (n * NOUT)) * e)
    g = np.zeros(SIZE, dtype=np.float32)
    g[OFF_W4:OFF_B4] = (dy.T @ h3).ravel()
    g[OFF_B4:SIZE] = dy.sum(axis=0)
    d3 = bf16((dy @ W4) * (h3 > 0))
    g[OFF_W3:OFF_B3] = (d3.T @ h2).ravel()
    g[OFF_B3:OFF_W4] = d3.sum(axis=0)
    d2 = bf16((d3 @ W3) * (h2 > 0))
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(axis=0)
    d1 = bf16((d2 @ W2) * (h1 > 0))
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(axis=0)
    return loss, g
