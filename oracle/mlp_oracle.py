"""NumPy oracle of the surrogate MLP — test infrastructure only.

Forward and backward of features -> 512 -> 256 -> 1 (ReLU, MSE loss) in
float64, optionally rounding to bfloat16 at the points where the CUDA
implementation (``brkga_fft2_b200/csrc/brkga_surrogate.cu``) stores bf16
operands for its tensor-core GEMMs, plus the feature extraction and Adam.
Used to check the GPU gradients; ``loss`` and ``grads`` with ``bf16=False``
are themselves checked against central finite differences.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _r(x, on):
    return bf16(x) if on else np.asarray(x, np.float64)


def forward(p, X, bf=True):
    W1, W2 = _r(p["W1"], bf), _r(p["W2"], bf)
    A1 = np.maximum(X @ W1.T + p["b1"], 0.0)
    H1 = _r(A1, bf)
    A2 = np.maximum(H1 @ W2.T + p["b2"], 0.0)
    y = A2 @ p["w3"] + p["b3"][0]
    return y, (A1, H1, A2)


def loss(p, X, t, n, bf=False):
    y, _ = forward(p, X, bf)
    e = (y - t)[:n]
    return float((e * e).mean())


def grads(p, X, t, n, bf=True):
    """Gradients of the mean squared error over the first n rows."""
    y, (A1, H1, A2) = forward(p, X, bf)
    dy = np.zeros_like(y)
    dy[:n] = 2.0 * (y[:n] - t[:n]) / n
    g = {"w3": A2.T @ dy, "b3": np.array([dy.sum()])}
    dZ2 = dy[:, None] * p["w3"][None, :] * (A2 > 0)
    g["b2"] = dZ2.sum(axis=0)
    dZ2q = _r(dZ2, bf)
    g["W2"] = dZ2q.T @ H1
    dH1 = dZ2q @ _r(p["W2"], bf)
    dZ1 = dH1 * (A1 > 0)
    g["b1"] = dZ1.sum(axis=0)
    g["W1"] = _r(dZ1, bf).T @ X
    return g


def numeric_grads(p, X, t, n, names=("W1", "b1", "W2", "b2", "w3", "b3"), eps=1e-6, samples=12, seed=0):
    """Central differences of the float64 loss at a few random coordinates of each parameter."""
    rng = np.random.default_rng(seed)
    out = {}
    for name in names:
        arr = p[name]
        idx = [tuple(int(rng.integers(0, s)) for s in arr.shape) for _ in range(samples)]
        vals = []
        for ix in idx:
            old = arr[ix]
            arr[ix] = old + eps
            lp = loss(p, X, t, n)
            arr[ix] = old - eps
            lm = loss(p, X, t, n)
            arr[ix] = old
            vals.append((lp - lm) / (2 * eps))
        out[name] = (idx, np.array(vals))
    return out


def adam(w, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v


def features(packed, chrom, in_pad):
    """Feature rows of host chromosomes [P, 2N] as the CUDA kernel builds them (bf16 values)."""
    a = packed.arrays
    N, M, T = packed.n_genes, packed.n_machines, packed.n_types
    thr = a["thresholds"][: max(M - 1, 0)]
    pt = a["proc_time"].reshape(M, T)
    pth = a["proc_time_height"].reshape(M, T)
    inv_pt = np.float32(1.0 / pt.max()) if pt.max() > 0 else np.float32(1)
    inv_pth = np.float32(1.0 / pth.max()) if pth.max() > 0 else np.float32(1)
    gt = a["gene_type"]
    out = np.zeros((chrom.shape[0], in_pad), np.float64)
    for r, ch in enumerate(np.asarray(chrom, np.float32)):
        sv, mv = ch[:N], ch[N:]
        if M <= 1:
            mach = np.zeros(N, np.int64)
        else:
            t32 = thr.astype(np.float32) if packed.threshold_mode == 0 else thr
            vals = mv if packed.threshold_mode == 0 else mv.astype(np.float64)
            mach = np.full(N, M - 1, np.int64)
            for m in range(M - 2, -1, -1):
                mach = np.where(vals <= t32[m], m, mach)
            mach = np.where(np.isnan(mv), M, mach)
        svc = np.where(sv == 0, np.float32(0), sv)
        order = np.lexsort((np.arange(N), svc, mach))
        area = np.zeros(M, np.float32)
        load = np.zeros(M, np.float32)
        for j in order:  # per-machine sums in decode order
            m = mach[j]
            if m < M:
                t = gt[j]
                area[m] += np.float32(a["part_area"][t] / a["bin_area"][m])
                load[m] += np.float32(pt[m, t]) * inv_pt
        f = np.zeros(in_pad, np.float32)
        mscale = np.float32(1.0 / (M - 1)) if M > 1 else np.float32(0)
        for pos, j in enumerate(order):
            m = mach[j]
            if m >= M:
                continue
            t = gt[j]
            f[3 * pos] = np.float32(m) * mscale
            f[3 * pos + 1] = np.float32(pt[m, t]) * inv_pt
            f[3 * pos + 2] = np.float32(pth[m, t]) * inv_pth
        f[3 * N:3 * N + 2 * M:2] = area
        f[3 * N + 1:3 * N + 2 * M:2] = load
        out[r] = bf16(f)
    return out


def order_features(packed, chrom, in_pad):
    """Order feature rows (BRKGA_SURROGATE_FEATURES_ORDER) of host chromosomes:
    the parts sorted by sequencing key (ties by gene index, machine keys
    ignored), per part its key, area / largest part area and height time on
    machine 0 / largest height time, as bf16 values."""
    a = packed.arrays
    N, M, T = packed.n_genes, packed.n_machines, packed.n_types
    pth = a["proc_time_height"].reshape(M, T)
    inv_pth = np.float32(1.0 / pth.max()) if pth.max() > 0 else np.float32(1)
    inv_area = np.float32(1.0 / a["part_area"].max())
    gt = a["gene_type"]
    out = np.zeros((chrom.shape[0], in_pad), np.float64)
    for r, ch in enumerate(np.asarray(chrom, np.float32)):
        sv = ch[:N]
        svc = np.where(sv == 0, np.float32(0), sv)
        order = np.lexsort((np.arange(N), svc))
        f = np.zeros(in_pad, np.float32)
        for pos, j in enumerate(order):
            t = gt[j]
            f[3 * pos] = ch[j]
            f[3 * pos + 1] = np.float32(a["part_area"][t]) * inv_area
            f[3 * pos + 2] = np.float32(pth[0, t]) * inv_pth
        out[r] = bf16(f)
    return out
