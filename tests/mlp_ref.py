"""numpy restatement of the learned-bracket network (psod_b200/csrc/psod_learn.cu).

Test infrastructure: the GPU forward and gradient kernels are checked
against ``forward`` / ``gradient`` here.  With ``emulate=True`` the same
bfloat16 rounding points as the kernels are applied (inputs, weights, hidden
activations, output and hidden gradients); products are then accumulated in
float64, so the only differences left are the kernels' FP32 accumulation
order.  With ``emulate=False`` everything is float64, which is what the
finite-difference check differentiates.
"""

from __future__ import annotations

import numpy as np

NF, IN, HID, NOUT, OUTP = 10, 16, 64, 2, 8
OW1 = 0
OB1 = OW1 + HID * IN
OW2 = OB1 + HID
OB2 = OW2 + HID * HID
OW3 = OB2 + HID
OB3 = OW3 + OUTP * HID
NPARAM = OB3 + OUTP
NNORM = 2 * IN + 2 * NOUT
NBLOB = NNORM + NPARAM


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def random_blob(seed: int, scale: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = np.zeros(NBLOB, np.float32)
    b[0:NF] = rng.normal(0, 1, NF)                       # mu_x
    b[IN : IN + IN] = 1.0
    b[IN : IN + NF] = rng.uniform(0.5, 2.0, NF)          # sigma_x
    b[2 * IN : 2 * IN + NOUT] = rng.normal(0, 1, NOUT)   # mu_y
    b[2 * IN + NOUT : NNORM] = rng.uniform(0.5, 2.0, NOUT)
    p = b[NNORM:]
    w1 = np.zeros((HID, IN), np.float32)
    w1[:, :NF] = rng.uniform(-1, 1, (HID, NF)) * np.sqrt(6 / NF) * scale
    p[OW1:OB1] = w1.ravel()
    p[OB1:OW2] = rng.normal(0, 0.1, HID)
    p[OW2:OB2] = (rng.uniform(-1, 1, HID * HID) * np.sqrt(6 / HID) * scale).astype(np.float32)
    p[OB2:OW3] = rng.normal(0, 0.1, HID)
    w3 = np.zeros((OUTP, HID), np.float32)
    w3[:NOUT] = rng.uniform(-1, 1, (NOUT, HID)) * np.sqrt(6 / HID) * 0.5
    p[OW3:OB3] = w3.ravel()
    p[OB3 : OB3 + NOUT] = rng.normal(0, 0.1, NOUT)
    return b


def unpack(blob):
    b = np.asarray(blob)
    if b.dtype != np.float64:
        b = b.astype(np.float32)
    mux, sgx = b[0:IN], b[IN : 2 * IN]
    muy, sgy = b[2 * IN : 2 * IN + NOUT], b[2 * IN + NOUT : NNORM]
    p = b[NNORM:]
    return dict(
        mux=mux, sgx=sgx, muy=muy, sgy=sgy,
        w1=p[OW1:OB1].reshape(HID, IN), b1=p[OB1:OW2],
        w2=p[OW2:OB2].reshape(HID, HID), b2=p[OB2:OW3],
        w3=p[OW3:OB3].reshape(OUTP, HID), b3=p[OB3:NPARAM],
    )


def standardize_x(m, x):
    x = np.asarray(x, np.float32)
    xs = np.zeros((x.shape[0], IN), np.float32)
    xs[:, :NF] = (x[:, :NF] - m["mux"][:NF]) / m["sgx"][:NF]  # float32, as the kernel
    return xs


def _forward(m, x, emulate):
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    X = r(standardize_x(m, x)).astype(np.float64)
    W1, W2, W3 = (r(m[k]).astype(np.float64) for k in ("w1", "w2", "w3"))
    pre1 = X @ W1.T + m["b1"]
    H1 = np.maximum(pre1, 0.0)
    if emulate:
        H1 = bf16(H1.astype(np.float32)).astype(np.float64)
    pre2 = H1 @ W2.T + m["b2"]
    H2 = np.maximum(pre2, 0.0)
    if emulate:
        H2 = bf16(H2.astype(np.float32)).astype(np.float64)
    y = (H2 @ W3.T + m["b3"])[:, :NOUT]
    return X, W1, W2, W3, H1, H2, y


def forward(blob, x, emulate: bool = True) -> np.ndarray:
    """Outputs in original units: y * sigma_y + mu_y."""
    m = unpack(blob)
    y = _forward(m, x, emulate)[-1]
    return y * m["sgy"] + m["muy"]


def gradient(blob, x, t, emulate: bool = True):
    """(gradient in the padded parameter layout, loss) of
    0.5 * sum |y_std - t_std|^2 / n."""
    m = unpack(blob)
    n = x.shape[0]
    X, W1, W2, W3, H1, H2, y = _forward(m, x, emulate)
    ts = ((np.asarray(t, np.float32) - m["muy"]) / m["sgy"]).astype(np.float64)
    diff = y - ts
    loss = 0.5 * float((diff**2).sum()) / n
    dY = np.zeros((n, OUTP))
    dY[:, :NOUT] = diff / n
    if emulate:
        dY = bf16(dY.astype(np.float32)).astype(np.float64)
    dH2 = (dY @ W3) * (H2 > 0)
    if emulate:
        dH2 = bf16(dH2.astype(np.float32)).astype(np.float64)
    dH1 = (dH2 @ W2) * (H1 > 0)
    if emulate:
        dH1 = bf16(dH1.astype(np.float32)).astype(np.float64)
    g = np.zeros(NPARAM)
    g[OW1:OB1] = (dH1.T @ X).ravel()
    g[OB1:OW2] = dH1.sum(0)
    g[OW2:OB2] = (dH2.T @ H1).ravel()
    g[OB2:OW3] = dH2.sum(0)
    g[OW3:OB3] = (dY.T @ H2).ravel()
    g[OB3:NPARAM] = dY.sum(0)
    return g, loss


def loss64(blob, x, t) -> float:
    m = unpack(blob)
    y = _forward(m, x, False)[-1]
    ts = ((np.asarray(t, np.float32) - m["muy"]) / m["sgy"]).astype(np.float64)
    return 0.5 * float(((y - ts) ** 2).sum()) / x.shape[0]
