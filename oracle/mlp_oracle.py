"""CPU oracle of the learned cost model (test infrastructure only).

A numpy float64 restatement of the library's 5 -> 64 -> 64 -> 1 ReLU MLP and of its job
features, used to check the CUDA forward/backward kernels (g3sa_b200/csrc/g3x_model.cu).
The model has no counterpart in the reference; this file is its specification.

Parameter layout (4,609 floats): W1[64][5] | b1[64] | W2[64][64] | b2[64] | W3[64] | b3.
"""
import numpy as np

F, H = 5, 64
OFF = {"W1": 0, "b1": H * F, "W2": H * F + H, "b2": H * F + H + H * H,
       "W3": H * F + 2 * H + H * H, "b3": H * F + 3 * H + H * H}
NPARAMS = OFF["b3"] + 1
assert NPARAMS == 4609


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF["W1"]:OFF["b1"]].reshape(H, F), p[OFF["b1"]:OFF["W2"]],
            p[OFF["W2"]:OFF["b2"]].reshape(H, H), p[OFF["b2"]:OFF["W3"]],
            p[OFF["W3"]:OFF["b3"]], p[OFF["b3"]])


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    A1 = X @ W1.T + b1
    H1 = np.maximum(A1, 0)
    A2 = H1 @ W2.T + b2
    H2 = np.maximum(A2, 0)
    Y = H2 @ W3 + b3
    return Y, (X, H1, H2)


def loss_and_grad(p, X, T):
    """Mean squared error over the batch and its gradient (flat, library layout)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Y, (X, H1, H2) = forward(p, X)
    T = np.asarray(T, np.float64)
    B = len(T)
    e = Y - T
    loss = float(np.mean(e * e))
    dY = 2 * e / B
    g = np.zeros(NPARAMS)
    g[OFF["W3"]:OFF["b3"]] = dY @ H2
    g[OFF["b3"]] = dY.sum()
    dH2 = np.outer(dY, W3) * (H2 > 0)
    g[OFF["W2"]:OFF["b2"]] = (dH2.T @ H1).ravel()
    g[OFF["b2"]:OFF["W3"]] = dH2.sum(0)
    dH1 = (dH2 @ W2) * (H1 > 0)
    g[OFF["W1"]:OFF["b1"]] = (dH1.T @ X).ravel()
    g[OFF["b1"]:OFF["W2"]] = dH1.sum(0)
    return loss, g


def features(jobs, u8):
    """Per job: qlen/128, tlen/256, h0/64, and the ungapped extension along the seed's diagonal
    over the first min(qlen, tlen) bases -- from h0, +1 per identical base pair, -4 per other
    pair (N on either side counts as different) -- as its best score / 64 and the number of
    bases at which that score is first reached / 128 (0 when it is h0 itself)."""
    out = np.zeros((len(jobs), F), np.float64)
    for k, jb in enumerate(jobs):
        q = u8[jb["q_off"]:jb["q_off"] + jb["qlen"]]
        t = u8[jb["t_off"]:jb["t_off"] + jb["tlen"]]
        if jb["flags"] & 1:
            q = q[::-1]
        if jb["flags"] & 2:
            t = t[::-1]
        kk = min(len(q), len(t))
        same = (q[:kk] == t[:kk]) & (q[:kk] < 4) & (t[:kk] < 4)
        s = int(jb["h0"]) + np.concatenate([[0], np.cumsum(np.where(same, 1, -4))])
        at = int(np.argmax(s))
        out[k] = (jb["qlen"] / 128, jb["tlen"] / 256, jb["h0"] / 64, s[at] / 64, at / 128)
    return out
