"""Float64 CPU restatement of the cost model (test infrastructure): features, forward pass
and analytic gradients of the mean squared error, with fp16 rounding applied at the same
points as the GPU kernels (W1, W2 and the hidden activations H1, H2, dZ2, dZ1 are fp16
operands of the tensor-core GEMMs; everything else is accumulated in higher precision)."""
import numpy as np

IN, H = 112, 128
KW1, KB1 = 0, IN * H
KW2 = KB1 + H
KB2 = KW2 + H * H
KW3 = KB2 + H
KB3 = KW3 + H
NPARAMS = KB3 + 1
C, A = 0.7978845608028654, 0.044715


def f16(x):
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C * (x + A * x ** 3)))


def gelu_grad(x):
    th = np.tanh(C * (x + A * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * C * (1.0 + 3.0 * A * x * x)


def features(states):
    """Same encoding as the library (board-relative): free cells of each of the next 32 rows,
    the free-column and candidate masks centred on the board, then 6 scalars."""
    st = np.asarray(states)
    n = st["n"].astype(np.int64)
    row = st["row"].astype(np.int64)
    mask = ((np.int64(1) << n) - 1).astype(np.uint64)
    cols, ld, rd = (st[k].astype(np.uint64) for k in ("cols", "ldiag", "rdiag"))
    m32 = np.uint64(0xFFFFFFFF)
    nc = mask & ~cols & m32
    avail = nc & ~(ld | rd) & m32
    left = np.maximum(n - row, 0)
    shift = (16 - (n >> 1)).astype(np.uint64)
    pc = np.vectorize(lambda v: bin(int(v)).count("1"), otypes=[np.int64])
    X = np.zeros((len(st), IN), dtype=np.float64)
    if not len(st):
        return X
    look = np.zeros((len(st), 32), dtype=np.int64)
    for k in range(32):
        kk = np.uint64(k)
        cells = pc(nc & ~(((ld << kk) & m32) | (rd >> kk)))
        look[:, k] = np.where(k < left, cells, 0)
    X[:, 0:32] = look / 32.0
    bits = np.arange(32, dtype=np.uint64)
    X[:, 32:64] = ((((nc << shift) & m32)[:, None]) >> bits) & np.uint64(1)
    X[:, 64:96] = ((((avail << shift) & m32)[:, None]) >> bits) & np.uint64(1)
    X[:, 96] = left / 32.0
    X[:, 97] = pc(nc) / 32.0
    X[:, 98] = pc(avail) / 32.0
    X[:, 99] = n / 32.0
    X[:, 100] = row / 32.0
    X[:, 101] = look.sum(1) / 256.0
    return X


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[KW1:KB1].reshape(IN, H), p[KB1:KW2], p[KW2:KB2].reshape(H, H), p[KB2:KW3], p[KW3:KB3], p[KB3])


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    Zb1 = f16(X) @ f16(W1) + b1
    H1 = f16(gelu(Zb1))
    Zb2 = H1 @ f16(W2) + b2
    H2 = f16(gelu(Zb2))
    y = H2 @ w3 + b3
    return y, (Zb1, H1, Zb2, H2)


def loss_grad(p, X, t):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (Zb1, H1, Zb2, H2) = forward(p, X)
    B = len(t)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d
    g = np.zeros(NPARAMS)
    g[KW3:KB3] = H2.T @ dy / B
    g[KB3] = dy.sum() / B
    dZ2 = f16(dy[:, None] * w3[None, :] * gelu_grad(Zb2))
    g[KB2:KW3] = dZ2.sum(0) / B
    g[KW2:KB2] = (H1.T @ dZ2 / B).ravel()
    dH1 = dZ2 @ f16(W2).T
    dZ1 = f16(dH1 * gelu_grad(Zb1))
    g[KB1:KW2] = dZ1.sum(0) / B
    g[KW1:KB1] = (f16(X).T @ dZ1 / B).ravel()
    return loss, g
