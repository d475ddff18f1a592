"""NumPy restatement of the scheduler's cost-model MLP -- TEST INFRASTRUCTURE ONLY.

The checker for the CUDA forward/backward kernels of the learned scheduler
(the kernels in cupami_b200/csrc/k_costmodel.cuh).  Same parameter layout:
mu[NF] | inv_sigma[NF] | W1[H][NF] | b1[H] | w2[H] | b2 | y_mu | y_sigma.
"""

import numpy as np

NF, H = 16, 64
OFF_MU = 0
OFF_IS = NF
OFF_W1 = 2 * NF
OFF_B1 = OFF_W1 + H * NF
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H
OFF_YMU = OFF_B2 + 1
OFF_YSD = OFF_YMU + 1
N_PARAMS = OFF_YSD + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_MU:OFF_IS], p[OFF_IS:OFF_W1], p[OFF_W1:OFF_B1].reshape(H, NF), p[OFF_B1:OFF_W2],
            p[OFF_W2:OFF_B2], p[OFF_B2], p[OFF_YMU], p[OFF_YSD])


def forward(p, X, raw=True):
    mu, isd, W1, b1, w2, b2, ymu, ysd = unpack(p)
    x = (np.asarray(X, np.float64) - mu) * isd
    a = x @ W1.T + b1
    out = np.maximum(a, 0) @ w2 + b2
    return out * ysd + ymu if raw else out


def gradient(p, X, y):
    """Gradient of (1/2n) sum (f(x) - t)^2, t = (y - y_mu) / y_sigma; and the loss."""
    mu, isd, W1, b1, w2, b2, ymu, ysd = unpack(p)
    x = (np.asarray(X, np.float64) - mu) * isd
    t = (np.asarray(y, np.float64) - ymu) / (ysd if ysd != 0 else 1.0)
    a = x @ W1.T + b1
    r = np.maximum(a, 0)
    e = r @ w2 + b2 - t
    n = len(t)
    g = np.zeros(N_PARAMS)
    g[OFF_B2] = e.sum() / n
    g[OFF_W2:OFF_B2] = r.T @ e / n
    d = (e[:, None] * w2[None, :]) * (a > 0)
    g[OFF_B1:OFF_W2] = d.sum(axis=0) / n
    g[OFF_W1:OFF_B1] = (d.T @ x).reshape(-1) / n
    return g, 0.5 * float(e @ e) / n
