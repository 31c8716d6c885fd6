"""NumPy restatement of the gapped-stage cost model (8 -> 32 -> 32 -> 1 ReLU
MLP, mean squared error) used to check the CUDA training and inference
kernels.  TEST INFRASTRUCTURE ONLY."""
import numpy as np

FEAT, HID = 8, 32
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * FEAT
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID
PARAMS = OFF_B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(HID, FEAT), p[OFF_B1:OFF_W2],
            p[OFF_W2:OFF_B2].reshape(HID, HID), p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def loss_and_grad(p, X, Y):
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    n = len(Y)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    y, (z1, h1, z2, h2) = forward(p, X)
    d = y - Y
    loss = float((d * d).mean())
    dy = 2 * d / n
    g = np.zeros(PARAMS)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    dh2 = np.outer(dy, W3) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (dh1.T @ X).reshape(-1)
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    return loss, g
