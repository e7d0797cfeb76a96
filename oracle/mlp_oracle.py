"""CPU oracle of the learned con2prim seed network (test infrastructure).

numpy restatement of the forward and backward passes that
mhd-kh-instability_b200/csrc/cueva_train.cu runs on the GPU: the same
feature map, normalisation, bf16 rounding of the weights and biases, SiLU
layers 6 -> 64 -> 64 -> 64 -> 1 and mean-squared loss on the normalised
log(p/D).  The network has no counterpart in the reference; the oracle pins
the GPU gradients (checked in float64 here, against finite differences in
the CPU tests).
"""
import numpy as np

H, NIN = 64, 6
OFF = {}
_o = 0
for _name, _size in (("W1", H * NIN), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H),
                     ("W4", H), ("b4", 1)):
    OFF[_name] = (_o, _size)
    _o += _size
NPARAM = _o


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, rounded=True):
    w = {k: np.asarray(params[o:o + n], dtype=np.float64) for k, (o, n) in OFF.items()}
    if rounded:
        w = {k: bf16(np.asarray(params[o:o + n], dtype=np.float32)) for k, (o, n) in OFF.items()}
    w["W1"] = w["W1"].reshape(H, NIN)
    w["W2"] = w["W2"].reshape(H, H)
    w["W3"] = w["W3"].reshape(H, H)
    w["W4"] = w["W4"].reshape(1, H)
    return w


def features(cons):
    """cons (11, n): D, tau, Sx, Sy, Sz, Ex, Ey, Ez, Bx, By, Bz -> (n, 6):
    log D, log(Ef/M), log(M/D - 1), log(1+|B|^2/D), log(1+|E|^2/D), cos(S,B)
    with Sf = S - E x B, Ef = tau - (E^2+B^2)/2, M = sqrt(Ef^2 - |Sf|^2)."""
    D, tau = cons[0], cons[1]
    S, E, B = cons[2:5], cons[5:8], cons[8:11]
    S2, B2, E2 = (S * S).sum(0), (B * B).sum(0), (E * E).sum(0)
    SB = (S * B).sum(0)
    ExB = np.stack([E[1] * B[2] - E[2] * B[1], E[2] * B[0] - E[0] * B[2], E[0] * B[1] - E[1] * B[0]])
    Sf = S - ExB
    sfm = np.sqrt((Sf * Sf).sum(0))
    Ef = tau - 0.5 * (E2 + B2)
    M = np.sqrt(np.maximum((Ef - sfm) * (Ef + sfm), 0.0))
    den = np.sqrt(S2 * B2)
    f32 = np.float32
    f = np.stack([np.log(D.astype(f32)), np.minimum(np.log((Ef / np.maximum(M, 1e-300)).astype(f32)), 10.0),
                  np.log(np.maximum(M / D - 1.0, 1e-9).astype(f32)), np.log1p((B2 / D).astype(f32)),
                  np.log1p((E2 / D).astype(f32)),
                  np.where(den > 0, SB / np.where(den > 0, den, 1.0), 0.0)], axis=1)
    return f.astype(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward_backward(params, norm, cons, p):
    """Loss and gradient (flat, NPARAM) of the normalised-log-pressure MSE."""
    w = unpack(params)
    mu, sd, mu_y, sd_y = norm[:NIN], norm[NIN:2 * NIN], norm[2 * NIN], norm[2 * NIN + 1]
    X = (features(cons) - mu) / sd
    T = (np.log(p / cons[0]).astype(np.float32).astype(np.float64) - mu_y) / sd_y
    Z1 = X @ w["W1"].T + w["b1"]; A1 = silu(Z1)
    Z2 = A1 @ w["W2"].T + w["b2"]; A2 = silu(Z2)
    Z3 = A2 @ w["W3"].T + w["b3"]; A3 = silu(Z3)
    Y = (A3 @ w["W4"].T)[:, 0] + w["b4"][0]
    n = X.shape[0]
    loss = np.mean((Y - T) ** 2)
    dY = 2.0 * (Y - T) / n

    def dsilu(z):
        s = 1.0 / (1.0 + np.exp(-z))
        return s * (1.0 + z * (1.0 - s))

    g = {}
    g["W4"] = dY[None, :] @ A3
    g["b4"] = np.array([dY.sum()])
    dZ3 = (dY[:, None] @ w["W4"]) * dsilu(Z3)
    g["W3"] = dZ3.T @ A2; g["b3"] = dZ3.sum(0)
    dZ2 = (dZ3 @ w["W3"]) * dsilu(Z2)
    g["W2"] = dZ2.T @ A1; g["b2"] = dZ2.sum(0)
    dZ1 = (dZ2 @ w["W2"]) * dsilu(Z1)
    g["W1"] = dZ1.T @ X; g["b1"] = dZ1.sum(0)
    flat = np.zeros(NPARAM)
    for k, (o, nn) in OFF.items():
        flat[o:o + nn] = np.asarray(g[k]).ravel()
    return loss, flat


def loss_only(params_f64, norm, cons, p):
    """Loss with unrounded float64 parameters (finite-difference checks)."""
    w = unpack(params_f64, rounded=False)
    mu, sd, mu_y, sd_y = norm[:NIN], norm[NIN:2 * NIN], norm[2 * NIN], norm[2 * NIN + 1]
    X = (features(cons) - mu) / sd
    T = (np.log(p / cons[0]) - mu_y) / sd_y
    A = silu(X @ w["W1"].T + w["b1"])
    A = silu(A @ w["W2"].T + w["b2"])
    A = silu(A @ w["W3"].T + w["b3"])
    Y = (A @ w["W4"].T)[:, 0] + w["b4"][0]
    return np.mean((Y - T) ** 2)
