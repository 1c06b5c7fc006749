"""ORACLE (test infrastructure only): FP64 numpy restatement of the property-surrogate MLP's
forward pass, loss and gradients, used to check the library's own FP32 training kernels.

Network 1 -> 64 -> 64 -> 64 -> 4, tanh on the hidden layers, flat parameter layout
W1[64x1], b1[64], W2[64x64], b2[64], W3[64x64], b3[64], W4[4x64], b4[4] (W rows = outputs).
Loss = mean over the B*4 outputs of (y - t)^2.
"""
import numpy as np

H, NOUT = 64, 4
OFF = dict(W1=0, b1=64, W2=128, b2=128 + 4096, W3=128 + 4096 + 64, b3=128 + 2 * 4096 + 64,
           W4=128 + 2 * 4096 + 128, b4=128 + 2 * 4096 + 128 + 256)
NPARAM = OFF["b4"] + 4


def unpack(p):
    p = np.asarray(p, np.float64)
    return dict(W1=p[OFF["W1"]:OFF["b1"]].reshape(H, 1), b1=p[OFF["b1"]:OFF["W2"]],
                W2=p[OFF["W2"]:OFF["b2"]].reshape(H, H), b2=p[OFF["b2"]:OFF["W3"]],
                W3=p[OFF["W3"]:OFF["b3"]].reshape(H, H), b3=p[OFF["b3"]:OFF["W4"]],
                W4=p[OFF["W4"]:OFF["b4"]].reshape(NOUT, H), b4=p[OFF["b4"]:NPARAM])


def forward(p, x):
    w = unpack(p)
    x = np.asarray(x, np.float64).reshape(-1, 1)
    h1 = np.tanh(x @ w["W1"].T + w["b1"])
    h2 = np.tanh(h1 @ w["W2"].T + w["b2"])
    h3 = np.tanh(h2 @ w["W3"].T + w["b3"])
    y = h3 @ w["W4"].T + w["b4"]
    return y, (x, h1, h2, h3)


def loss_and_grad(p, x, t):
    w = unpack(p)
    y, (x, h1, h2, h3) = forward(p, x)
    t = np.asarray(t, np.float64).reshape(y.shape)
    n = y.size
    r = y - t
    loss = float(np.sum(r * r) / n)
    dy = 2.0 * r / n
    g = np.zeros(NPARAM)
    g[OFF["W4"]:OFF["b4"]] = (dy.T @ h3).ravel()
    g[OFF["b4"]:] = dy.sum(0)
    dz3 = (dy @ w["W4"]) * (1.0 - h3 * h3)
    g[OFF["W3"]:OFF["b3"]] = (dz3.T @ h2).ravel()
    g[OFF["b3"]:OFF["W4"]] = dz3.sum(0)
    dz2 = (dz3 @ w["W3"]) * (1.0 - h2 * h2)
    g[OFF["W2"]:OFF["b2"]] = (dz2.T @ h1).ravel()
    g[OFF["b2"]:OFF["W3"]] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * (1.0 - h1 * h1)
    g[OFF["W1"]:OFF["b1"]] = (dz1.T @ x).ravel()
    g[OFF["b1"]:OFF["W2"]] = dz1.sum(0)
    return loss, g
