"""CPU oracle of the flavor chooser's network -- TEST INFRASTRUCTURE ONLY.

A numpy (float64) restatement of the perceptron the library trains on the GPU
(vldb_voila_b200/csrc/mlp.cu): in -> hidden (ReLU) -> hidden (ReLU) -> out, masked mean
squared error, parameters flattened as W1[in][hidden], b1, W2[hidden][hidden], b2,
W3[hidden][out], b3.  Used only to check the GPU forward pass and gradients (and, by
finite differences, to check itself).  This part has no counterpart in the reference.
"""
import numpy as np


def unpack(params, n_in, n_hid, n_out):
    p = np.asarray(params, dtype=np.float64)
    shapes = [(n_in, n_hid), (n_hid,), (n_hid, n_hid), (n_hid,), (n_hid, n_out), (n_out,)]
    out, off = [], 0
    for s in shapes:
        n = int(np.prod(s))
        out.append(p[off:off + n].reshape(s))
        off += n
    assert off == p.size
    return out


def forward(params, X, n_in, n_hid, n_out):
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, n_hid, n_out)
    X = np.asarray(X, dtype=np.float64)
    H1 = np.maximum(X @ W1 + b1, 0.0)
    H2 = np.maximum(H1 @ W2 + b2, 0.0)
    return H2 @ W3 + b3, (X, H1, H2)


def loss_grad(params, X, T, mask, n_in, n_hid, n_out):
    """(loss, flattened gradient) of the masked mean squared error."""
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, n_hid, n_out)
    Y, (X, H1, H2) = forward(params, X, n_in, n_hid, n_out)
    T = np.asarray(T, dtype=np.float64)
    M = np.ones_like(T) if mask is None else np.asarray(mask, dtype=np.float64)
    denom = max(M.sum(), 1.0)
    D = Y - T
    loss = float((M * D * D).sum() / denom)
    dY = 2.0 * M * D / denom
    dW3 = H2.T @ dY
    db3 = dY.sum(axis=0)
    dH2 = (dY @ W3.T) * (H2 > 0)
    dW2 = H1.T @ dH2
    db2 = dH2.sum(axis=0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    dW1 = X.T @ dH1
    db1 = dH1.sum(axis=0)
    g = np.concatenate([a.reshape(-1) for a in (dW1, db1, dW2, db2, dW3, db3)])
    return loss, g
