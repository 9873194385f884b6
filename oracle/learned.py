"""TEST INFRASTRUCTURE ONLY: NumPy restatement of the learned preconditioner's forward and
backward passes, the checker of the GPU training and inference kernels.

Network (applied to a residual r of the Jacobi-scaled edge system S^, unit diagonal):
    h0_i = (r_i, 0, 0, 0)
    layer l = 0, 1, 2:   a = S^ h^l                                   (4 channels)
                         u_i = [h^l_i ; a_i]                          (8)
                         s_i = W1 bf16(u_i) + b1                      (32)
                         o_i = W2 bf16(relu(s_i)) + b2                (4)
                         h^{l+1}_i = h^l_i + o_i
    z_i = h3_i[0]
W1, W2 are rounded to bfloat16 (the tensor-core operands), b1, b2 and all accumulation are
FP32.  With W2 = 0 and b2 = 0 the network is the identity, i.e. Jacobi preconditioning.
Loss on one pair (r, e) with S^ e = r (e: the correction the plain solver needed):
    L = (z - e)' S^ (z - e) / (e' S^ e) = (z - e)' (S^ z - r) / (e' r)      (energy norm)
Parameter layout per layer (420 floats): W1 [32][8], b1 [32], W2 [4][32], b2 [4].
"""
import numpy as np

K = 4            # node state channels
H = 32           # MLP width
LAYERS = 3
PER_LAYER = H * 2 * K + H + K * H + K
N_PARAMS = LAYERS * PER_LAYER


QUANTIZE = True   # False: no bf16 rounding, all FP64 (finite-difference checks of the gradient)


def _ft():
    """Activation type: FP32 as on the GPU, FP64 for the unquantised self-checks."""
    return np.float32 if QUANTIZE else np.float64


def bf16(x):
    """Round to bfloat16 (nearest even) and back to float32."""
    if not QUANTIZE:
        return np.asarray(x, np.float64)
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, _ft())
    out = []
    for l in range(LAYERS):
        o = l * PER_LAYER
        W1 = w[o:o + H * 2 * K].reshape(H, 2 * K); o += H * 2 * K
        b1 = w[o:o + H]; o += H
        W2 = w[o:o + K * H].reshape(K, H); o += K * H
        b2 = w[o:o + K]
        out.append((W1, b1, W2, b2))
    return out


def init_weights(seed=0, scale=0.1):
    """W1 random, W2 = b2 = 0 (identity network), b1 = 0."""
    rng = np.random.default_rng(seed)
    w = np.zeros(N_PARAMS, np.float32)
    for l in range(LAYERS):
        o = l * PER_LAYER
        w[o:o + H * 2 * K] = rng.normal(0.0, scale, H * 2 * K)
    return w


def forward(S, r, w):
    """Returns z and the per-layer caches (h, u, s)."""
    S = S.astype(np.float64)
    ft = _ft()
    h = np.zeros((len(r), K), ft)
    h[:, 0] = r
    caches = []
    for (W1, b1, W2, b2) in unpack(w):
        a = (S @ h.astype(np.float64)).astype(ft)
        u = np.concatenate([h, a], axis=1)
        s = bf16(u) @ bf16(W1).T + b1
        hid = bf16(np.maximum(s, 0.0))
        o = hid @ bf16(W2).T + b2
        caches.append((h, u, s))
        h = (h + o).astype(ft)
    return h[:, 0].copy(), caches, h


def loss_and_grad(S, r, e, w):
    """Energy-norm loss of one pair and its gradient with respect to the FP32 parameters
    (straight-through through the bf16 rounding, as the GPU kernels do)."""
    z, caches, _ = forward(S, r, w)
    S64 = S.astype(np.float64)
    Sz = S64 @ z.astype(np.float64)
    er = float(np.dot(e, r))
    L = float(np.dot(z - e, Sz - r)) / er
    ft = _ft()
    gz = (2.0 * (Sz - r) / er).astype(ft)
    g = np.zeros((len(r), K), ft)
    g[:, 0] = gz
    grads = []
    for (W1, b1, W2, b2), (h, u, s) in zip(reversed(unpack(w)), reversed(caches)):
        hid = bf16(np.maximum(s, 0.0))
        dW2 = g.T @ hid
        db2 = g.sum(axis=0)
        g_hid = g @ bf16(W2)
        g_s = g_hid * (s > 0)
        dW1 = g_s.T @ bf16(u)
        db1 = g_s.sum(axis=0)
        g_u = g_s @ bf16(W1)
        g_h = g + g_u[:, :K] + (S64 @ g_u[:, K:].astype(np.float64)).astype(ft)
        grads.append(np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2]).astype(ft))
        g = g_h
    return L, np.concatenate(list(reversed(grads)))
