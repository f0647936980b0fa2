"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the learned coarse
correction's MLP (64 -> 256 -> 256 -> 32, ReLU, mean-squared-error loss) and
its backward pass, used to check the CUDA forward / backward kernels.
Parameter layout: W1 (64 x 256), b1, W2 (256 x 256), b2, W3 (256 x 32), b3."""
import numpy as np

F, H, O = 64, 256, 32


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    k = 0
    out = []
    for shape in [(F, H), (H,), (H, H), (H,), (H, O), (O,)]:
        n = int(np.prod(shape))
        out.append(p[k:k + n].reshape(shape))
        k += n
    return out


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    Y1 = np.maximum(X @ W1 + b1, 0.0)
    Y2 = np.maximum(Y1 @ W2 + b2, 0.0)
    return Y1, Y2, Y2 @ W3 + b3


def loss_and_grads(p, X, T):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    Y1, Y2, Y3 = forward(p, X)
    n = Y3.size
    loss = np.sum((Y3 - T) ** 2) / n
    d3 = 2.0 * (Y3 - T) / n
    gW3, gb3 = Y2.T @ d3, d3.sum(0)
    d2 = (d3 @ W3.T) * (Y2 > 0)
    gW2, gb2 = Y1.T @ d2, d2.sum(0)
    d1 = (d2 @ W2.T) * (Y1 > 0)
    gW1, gb1 = X.T @ d1, d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g, Y3
