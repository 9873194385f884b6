"""TEST INFRASTRUCTURE ONLY: NumPy restatement of the learned smoother network (no counterpart
in the reference), the checker of the GPU's forward and backward kernels (svn-export_b200/csrc/
smoother_nn.cu).  Never imported by the product.

The network reads the Jacobi-scaled edge system S^ (unit diagonal; off-diagonal o_ij) and
gives every row a weight w_i of the multigrid's fine-level smoother (Chebyshev on diag(w) S^):

  features x_i (8):  1, sum_j |o_ij|, max_j |o_ij|, sum_j o_ij, sum_j max(o_ij, 0),
                     (number of o_ij != 0) / 8, sum_j o_ij^2, [row has no o_ij != 0]
  h0 = relu(W0 x + b0)                                   8 -> 32
  layer l = 1..3:  a = A h_{l-1},  A_ij = |o_ij|         (message passing over the edge graph)
                   u = W_l [h_{l-1}; a] + b_l            64 -> 32
                   h_l = h_{l-1} + relu(u)
  z = w_out . h_3 + b_out,   w_i = exp(C tanh(z_i)),  C = ln 2  (w in [1/2, 2])

The dense layers' operands (weights, x, h, a) are rounded to bf16 as the tensor-core kernels
round them, with FP32 sums.  With w_out = 0 and b_out = 0 the network gives w = 1 (plain
smoothing), the untrained state.  Parameter layout (float32, PARAMS entries):
  W0 [32][8], b0 [32], then per layer W_l [32][64], b_l [32], then w_out [32], b_out [1].
"""
import numpy as np
import scipy.sparse as sp

WIDTH, NFEAT, LAYERS = 32, 8, 3
C_OUT = float(np.log(2.0))
PARAMS = WIDTH * NFEAT + WIDTH + LAYERS * (WIDTH * 2 * WIDTH + WIDTH) + WIDTH + 1


def bf16(a):
    """Round float32 to bf16 (round to nearest even) and back."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(theta):
    theta = np.asarray(theta)
    o = 0

    def take(*shape):
        nonlocal o
        n = int(np.prod(shape))
        v = theta[o:o + n].reshape(shape)
        o += n
        return v
    W0, b0 = take(WIDTH, NFEAT), take(WIDTH)
    layers = [(take(WIDTH, 2 * WIDTH), take(WIDTH)) for _ in range(LAYERS)]
    wout, bout = take(WIDTH), take(1)
    return W0, b0, layers, wout, bout


def features(Sh):
    """Row features of the Jacobi-scaled matrix (CSR, unit diagonal)."""
    Sh = sp.csr_matrix(Sh)
    n = Sh.shape[0]
    O = Sh - sp.diags(Sh.diagonal())
    O.eliminate_zeros()
    Oa = abs(O)
    x = np.zeros((n, NFEAT), np.float32)
    x[:, 0] = 1.0
    x[:, 1] = np.asarray(Oa.sum(axis=1)).ravel()
    x[:, 2] = np.asarray(Oa.max(axis=1).todense()).ravel()
    x[:, 3] = np.asarray(O.sum(axis=1)).ravel()
    x[:, 4] = np.asarray(O.maximum(0).sum(axis=1)).ravel()
    cnt = np.diff(O.indptr)
    x[:, 5] = cnt / 8.0
    x[:, 6] = np.asarray(O.multiply(O).sum(axis=1)).ravel()
    x[:, 7] = (cnt == 0).astype(np.float32)
    return x, Oa.tocsr().astype(np.float64)


def forward(theta, x, A, exact=False):
    """Weights w [n] and the activations the backward needs.  exact=True: FP64 throughout and
    no bf16 rounding (the smooth function whose derivative backward() computes, for finite
    differences)."""
    W0, b0, layers, wout, bout = unpack(theta)
    ft = np.float64 if exact else np.float32
    rnd = (lambda v: np.asarray(v, np.float64)) if exact else bf16
    u0 = rnd(x) @ rnd(W0).T + b0
    h = np.maximum(u0, 0.0).astype(ft)
    acts = {"u0": u0, "h": [h], "a": [], "u": []}
    for W, b in layers:
        a = (A @ h.astype(np.float64)).astype(ft)
        inp = np.concatenate([h, a], axis=1)
        u = rnd(inp) @ rnd(W).T + b
        h = (h + np.maximum(u, 0.0)).astype(ft)
        acts["a"].append(a)
        acts["u"].append(u)
        acts["h"].append(h)
    z = h @ np.asarray(wout, ft) + bout[0]
    w = np.exp(C_OUT * np.tanh(z))
    acts["z"] = z
    return w.astype(ft), acts


def backward(theta, x, A, acts, dw):
    """Gradient of a loss with respect to theta, given dL/dw [n] (bf16 roundings passed
    straight through)."""
    W0, b0, layers, wout, bout = unpack(theta)
    z = acts["z"].astype(np.float64)
    t = np.tanh(z)
    w = np.exp(C_OUT * t)
    dz = np.asarray(dw, np.float64) * w * C_OUT * (1.0 - t * t)
    h3 = acts["h"][-1].astype(np.float64)
    g_wout = h3.T @ dz
    g_bout = np.array([dz.sum()])
    dh = np.outer(dz, wout.astype(np.float64))
    g_layers = []
    for l in range(LAYERS - 1, -1, -1):
        W, b = layers[l]
        h_prev = acts["h"][l].astype(np.float64)
        a = acts["a"][l].astype(np.float64)
        u = acts["u"][l].astype(np.float64)
        du = dh * (u > 0)
        inp = np.concatenate([h_prev, a], axis=1)
        g_layers.append((du.T @ inp, du.sum(axis=0)))
        din = du @ W.astype(np.float64)
        dh = dh + din[:, :WIDTH] + A.T @ din[:, WIDTH:]
    g_layers.reverse()
    du0 = dh * (acts["u0"] > 0)
    g_W0 = du0.T @ x.astype(np.float64)
    g_b0 = du0.sum(axis=0)
    parts = [g_W0.ravel(), g_b0]
    for gW, gb in g_layers:
        parts += [gW.ravel(), gb]
    parts += [g_wout, g_bout]
    return np.concatenate(parts)


def init_params(seed=0):
    """Xavier-scaled random layers and a zero output layer (w = 1: the untrained network)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, np.sqrt(2.0 / (NFEAT + WIDTH)), WIDTH * NFEAT), np.zeros(WIDTH)]
    for _ in range(LAYERS):
        parts += [rng.normal(0.0, 0.5 * np.sqrt(2.0 / (3 * WIDTH)), WIDTH * 2 * WIDTH), np.zeros(WIDTH)]
    parts += [np.zeros(WIDTH), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)
