"""FP64 numpy restatement of the row-nnz predictor (5 -> 64 -> 64 -> 1, ReLU)
and of its mean-squared-error gradient — TEST INFRASTRUCTURE: the checker for
the CUDA training and inference kernels in bcl_b200/csrc/mlp.cu.  The
parameter layout is the kernels': W1[5][64] b1[64] W2[64][64] b2[64] w3[64] b3.
"""
import numpy as np

IN, H = 5, 64
SIZES = [("W1", (IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,)), ("b3", (1,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ w["W1"] + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(a2, 0)
    return h2 @ w["w3"] + w["b3"][0], (X, a1, h1, a2, h2)


def loss_and_grad(p, X, y):
    """L = mean((yhat - y)^2) and dL/dp in the kernels' layout."""
    w = unpack(p)
    yhat, (X, a1, h1, a2, h2) = forward(p, X)
    n = X.shape[0]
    err = yhat - np.asarray(y, dtype=np.float64)
    g = 2.0 * err / n
    d2 = np.outer(g, w["w3"]) * (a2 > 0)
    d1 = (d2 @ w["W2"].T) * (a1 > 0)
    grads = {"W1": X.T @ d1, "b1": d1.sum(0), "W2": h1.T @ d2, "b2": d2.sum(0), "w3": h2.T @ g,
             "b3": np.array([g.sum()])}
    flat = np.concatenate([grads[name].ravel() for name, _ in SIZES])
    return float(np.mean(err ** 2)), flat
