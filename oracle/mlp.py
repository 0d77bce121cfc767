"""CPU restatement of the learned-proposal MLP -- TEST INFRASTRUCTURE ONLY.

Forward pass, grouped softmax cross-entropy and back-propagation of the
scoring network in float64 numpy, in the parameter layout of the device
kernels (W1[44][128], b1, W2[128][128], b2, w3[128], b3); used to check the
device gradients.
"""
import numpy as np

IN, HID = 44, 128
SIZES = [("W1", IN * HID), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("w3", HID), ("b3", 1)]
N_PARAMS = sum(n for _, n in SIZES)


def unpack(p):
    out, o = {}, 0
    for k, n in SIZES:
        out[k] = np.asarray(p[o:o + n], dtype=np.float64)
        o += n
    out["W1"] = out["W1"].reshape(IN, HID)
    out["W2"] = out["W2"].reshape(HID, HID)
    return out


def scores(p, X):
    q = unpack(p)
    H1 = np.maximum(X @ q["W1"] + q["b1"], 0)
    H2 = np.maximum(H1 @ q["W2"] + q["b2"], 0)
    return H2 @ q["w3"] + q["b3"][0], H1, H2


def loss_and_grad(p, X, off, labels):
    X = np.asarray(X, dtype=np.float64)
    q = unpack(p)
    s, H1, H2 = scores(p, X)
    G = len(labels)
    ds = np.zeros_like(s)
    loss = 0.0
    for g in range(G):
        a, b = off[g], off[g + 1]
        z = s[a:b] - s[a:b].max()
        pr = np.exp(z) / np.exp(z).sum()
        loss -= np.log(pr[labels[g]])
        d = pr.copy()
        d[labels[g]] -= 1.0
        ds[a:b] = d / G
    gw3 = H2.T @ ds
    gb3 = np.array([ds.sum()])
    dH2 = np.outer(ds, q["w3"]) * (H2 > 0)
    gW2 = H1.T @ dH2
    gb2 = dH2.sum(0)
    dH1 = (dH2 @ q["W2"].T) * (H1 > 0)
    gW1 = X.T @ dH1
    gb1 = dH1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, gb3])
    return loss / G, grad
