"""FP64 numpy reference of the learned guide (TEST INFRASTRUCTURE ONLY).

Restates, in double precision, what research_b200/csrc/mlp_guide.cu computes
on the tensor cores: the input encoding, the 80-64-64-64-64-48 ReLU network,
the 8-lobe vMF mixture head, the weighted negative log-likelihood and its
gradient with respect to every parameter (with the same weight clamping,
normalisation and loss scale). The learned guide has no counterpart in the
reference renderer; this file is the checker for its forward and backward
passes.
"""
import numpy as np

LAYERS = [(80, 64), (64, 64), (64, 64), (64, 64), (64, 48)]
LOSS_SCALE = 1024.0
PARAM_COUNT = sum(o * i + o for i, o in LAYERS)


def unpack(params):
    out, k = [], 0
    for i, o in LAYERS:
        W = params[k:k + o * i].reshape(o, i); k += o * i
        b = params[k:k + o]; k += o
        out.append((W, b))
    return out


def encode(pos, n, wo, bmin, bmax):
    x = np.clip((pos - bmin) / (bmax - bmin), 0.0, 1.0)
    f = np.zeros((len(pos), 80))
    for a in range(3):
        for k in range(12):
            f[:, a * 24 + k] = np.sin(np.pi * 2.0 ** k * x[:, a])
            f[:, a * 24 + 12 + k] = np.cos(np.pi * 2.0 ** k * x[:, a])
    f[:, 72:75] = n
    f[:, 75:78] = wo
    return f


def forward(params, F):
    acts = [F]
    x = F
    for l, (W, b) in enumerate(unpack(params)):
        z = x @ W.T + b
        x = np.maximum(z, 0.0) if l < len(LAYERS) - 1 else z
        acts.append(x)
    return x, acts


def softplus(x):
    return np.where(x > 20, x, np.log1p(np.exp(np.minimum(x, 20))))


def mixture(raw):
    r = raw[:, :40].reshape(-1, 8, 5)
    v = r[:, :, :3]
    ln = np.maximum(np.linalg.norm(v, axis=2, keepdims=True), 1e-6)
    mu = v / ln
    kappa = np.minimum(softplus(r[:, :, 3]) + 0.1, 1000.0)
    lg = r[:, :, 4] - r[:, :, 4].max(axis=1, keepdims=True)
    pi = np.exp(lg) / np.exp(lg).sum(axis=1, keepdims=True)
    return mu, kappa, pi, ln[:, :, 0]


def nll_and_grad(raw, om):
    """-log p(om) under the mixture and d(-log p)/d(raw) (FP64)."""
    mu, kappa, pi, ln = mixture(raw)
    cosw = np.einsum("bjk,bk->bj", mu, om)
    lognorm = np.log(kappa) - np.log(2 * np.pi) - np.log1p(-np.exp(-2 * kappa))
    lq = np.log(np.maximum(pi, 1e-30)) + lognorm + kappa * (cosw - 1)
    lmax = lq.max(axis=1, keepdims=True)
    logp = lmax[:, 0] + np.log(np.exp(lq - lmax).sum(axis=1))
    gam = np.exp(lq - logp[:, None])
    g = np.zeros_like(raw)
    cv = -gam * kappa / ln
    gv = cv[:, :, None] * (om[:, None, :] - cosw[:, :, None] * mu)
    e2 = np.exp(-2 * kappa)
    dk = -gam * (1 / kappa - 2 * e2 / (1 - e2) + cosw - 1)
    dk = np.where(softplus(raw[:, :40].reshape(-1, 8, 5)[:, :, 3]) + 0.1 > 1000, 0.0, dk)
    sig = 1 / (1 + np.exp(-raw[:, :40].reshape(-1, 8, 5)[:, :, 3]))
    G = np.zeros((len(raw), 8, 5))
    G[:, :, :3] = gv
    G[:, :, 3] = dk * sig
    G[:, :, 4] = pi - gam
    g[:, :40] = G.reshape(-1, 40)
    return -logp, g


def batch_weights(w):
    clampv = 20.0 * w.mean()
    wc = np.minimum(w, clampv)
    return wc / wc.sum()


def loss_and_grad(params, F, om, w):
    """Weighted NLL (normalised weights) and its loss-scaled parameter gradient."""
    raw, acts = forward(params, F)
    wn = batch_weights(w)
    nll, g = nll_and_grad(raw, om)
    dz = g * (wn * LOSS_SCALE)[:, None]
    grads = []
    Ws = unpack(params)
    for l in range(len(LAYERS) - 1, -1, -1):
        W, _ = Ws[l]
        dW = dz.T @ acts[l]
        db = dz.sum(axis=0)
        grads.append((dW, db))
        if l > 0:
            dx = dz @ W
            dz = dx * (acts[l] > 0)
    grads = grads[::-1]
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return float((wn * nll).sum()), flat
