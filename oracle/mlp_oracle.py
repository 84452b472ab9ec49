"""CPU restatement (numpy, float64 arithmetic) of the troubled-cell network
and its gradients.  TEST INFRASTRUCTURE ONLY: the checker for the tensor-core
kernels of finess_b200/csrc/fin_mlp.cu.

Two forms:
* ``forward_emulated`` / ``grads_emulated`` round to BF16 exactly where the
  device does (inputs, the layer-1 activations, the weights and the layer-1
  bias, back-propagated activation gradients; the layer-2 activations enter
  the FP32 output layer unrounded), so they agree with the device to FP32
  accumulation error and the hardware tanh approximation;
* ``forward_exact`` / ``grads_exact`` have no rounding, for finite-difference
  checks of the back-propagation itself.
Parameter layout: W1[32][20], b1[32], W2[32][32], b2[32], w3[32], b3.
"""
import numpy as np

NIN, NH = 20, 32
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even), returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    W1 = P[OFF_W1:OFF_B1].reshape(NH, NIN)
    b1 = P[OFF_B1:OFF_W2]
    W2 = P[OFF_W2:OFF_B2].reshape(NH, NH)
    b2 = P[OFF_B2:OFF_W3]
    w3 = P[OFF_W3:OFF_B3]
    b3 = P[OFF_B3]
    return W1, b1, W2, b2, w3, b3


# GELU in its tanh form (Hendrycks & Gimpel, arXiv:1606.08415, eq. for the
# tanh approximation): gelu(x) = x/2 (1 + tanh(k0 x + k1 x^3)).
GK0 = np.sqrt(2.0 / np.pi)
GK1 = GK0 * 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(x * (GK0 + GK1 * x * x)))


def gelu_grad(x):
    t = np.tanh(x * (GK0 + GK1 * x * x))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * (GK0 + 3.0 * GK1 * x * x)


def _forward(P, X, rnd):
    W1, b1, W2, b2, w3, b3 = unpack(P)
    r = bf16 if rnd else (lambda v: np.asarray(v, dtype=np.float64))
    xb = r(X)
    a1 = xb @ r(W1).T + r(b1)
    g1 = r(gelu(a1))
    a2 = g1 @ r(W2).T + b2
    g2 = gelu(a2)
    z = g2 @ r(w3) + b3
    return xb, a1, g1, a2, g2, z


def forward_emulated(P, X):
    return _forward(P, X, True)[-1]


def forward_exact(P, X):
    return _forward(P, X, False)[-1]


def _grads(P, X, y, pos_weight, rnd):
    W1, b1, W2, b2, w3, b3 = unpack(P)
    r = bf16 if rnd else (lambda v: np.asarray(v, dtype=np.float64))
    xb, a1, g1, a2, g2, z = _forward(P, X, rnd)
    n = X.shape[0]
    y = np.asarray(y, dtype=np.float64)
    wgt = np.where(y > 0.5, pos_weight, 1.0)
    sp = np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))
    loss = np.sum(wgt * (sp - y * z))
    p = 1.0 / (1.0 + np.exp(-z))
    dz = wgt * (p - y) / n
    dh2 = (dz[:, None] * r(w3)[None, :]) * gelu_grad(a2)
    dh2b = r(dh2)
    dg1 = dh2b @ r(W2)
    dh1 = dg1 * gelu_grad(a1)
    dh1b = r(dh1)
    G = np.zeros(NPARAM)
    G[OFF_W1:OFF_B1] = (dh1b.T @ xb).ravel()
    G[OFF_B1:OFF_W2] = dh1.sum(0)
    G[OFF_W2:OFF_B2] = (dh2b.T @ g1).ravel()
    G[OFF_B2:OFF_W3] = dh2.sum(0)
    G[OFF_W3:OFF_B3] = (dz[:, None] * g2).sum(0)
    G[OFF_B3] = dz.sum()
    return G, loss


def grads_emulated(P, X, y, pos_weight=1.0):
    return _grads(P, X, y, pos_weight, True)


def grads_exact(P, X, y, pos_weight=1.0):
    return _grads(P, X, y, pos_weight, False)


def loss_exact(P, X, y, pos_weight=1.0):
    z = forward_exact(P, X)
    y = np.asarray(y, dtype=np.float64)
    wgt = np.where(y > 0.5, pos_weight, 1.0)
    sp = np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))
    return np.sum(wgt * (sp - y * z)) / X.shape[0]


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    P = np.zeros(NPARAM)
    P[OFF_W1:OFF_B1] = rng.uniform(-1, 1, NH * NIN) * np.sqrt(6.0 / NIN)
    P[OFF_W2:OFF_B2] = rng.uniform(-1, 1, NH * NH) * np.sqrt(6.0 / NH)
    P[OFF_W3:OFF_B3] = rng.uniform(-1, 1, NH) * np.sqrt(6.0 / NH)
    P[OFF_B1:OFF_W2] = rng.normal(0, 0.1, NH)
    P[OFF_B2:OFF_W3] = rng.normal(0, 0.1, NH)
    return P
