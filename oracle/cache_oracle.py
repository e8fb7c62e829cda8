"""ORACLE — test infrastructure only.  FP64 numpy restatement of the neural
cache (multiresolution hash-grid encoding + ReLU MLP) and its gradient, used as
the checker of the CUDA cache kernels.

The reference's cache is tiny-cuda-nn (NVlabs/tiny-cuda-nn, fetched from
`master` without a pin by scripts/fetch_tcnn.py:24-25; not vendored), called
at src/tools/eval_tcnn_nc_wos.cu:747-759.  Its arithmetic is restated here
from the published algorithm (Mueller et al., "Instant Neural Graphics
Primitives with a Multiresolution Hash Encoding", SIGGRAPH 2022): parity with
tiny-cuda-nn itself is unpinned (no reference test checks cache outputs).

Parameter layout (shared with the CUDA cache): [grid | mlp], grid = levels in
order, each level `table_size` entries x 2 features; mlp = W_in [W x in_dim]
(row = output neuron), hidden W_h [W x W] (hidden-1 of them), w_out [W],
zero padding to a multiple of 8.
"""
from __future__ import annotations

import math

import numpy as np

PRIMES = (1, 2654435761, 805459861)


def layout(n_levels=16, log2_T=19, base_res=16.0, max_res=2048.0, per_level_scale=0.0, width=64, hidden=2,
           resolutions=None):
    """Level / parameter layout.  resolutions: optional explicit N_l per level
    (the float rounding of floor(N_min * b^l) is otherwise recomputed here)."""
    b = per_level_scale
    if not b > 0:
        b = math.exp((math.log(np.float32(max_res)) - math.log(np.float32(base_res))) / (n_levels - 1)) if n_levels > 1 else 1.0
    b = float(np.float32(b))
    T = 1 << log2_T
    levels = []
    off = 0
    for l in range(n_levels):
        res = int(resolutions[l]) if resolutions is not None else \
            int(math.floor(np.float32(base_res) * np.float32(np.float32(b) ** np.float32(l))))
        dense = (res + 1) ** 3
        size = ((dense + 7) // 8) * 8 if dense <= T else T
        levels.append({"res": res, "dense": dense <= T, "size": size, "offset": off})
        off += size
    in_dim = 16 if n_levels * 2 <= 16 else 32
    o = 0
    mlp = {"w_in": o}
    o += width * in_dim
    mlp["w_hid"] = []
    for _ in range(hidden - 1):
        mlp["w_hid"].append(o)
        o += width * width
    mlp["w_out"] = o
    o += width
    mlp["total"] = (o + 7) // 8 * 8
    return {"levels": levels, "grid_params": off * 2, "in_dim": in_dim, "width": width, "hidden": hidden,
            "mlp": mlp, "scale": b}


def _corner_index(lv, x, y, z):
    if lv["dense"]:
        s = lv["res"] + 1
        return x + s * (y + s * z)
    h = (x.astype(np.uint64) * PRIMES[0]) ^ (y.astype(np.uint64) * PRIMES[1]) ^ (z.astype(np.uint64) * PRIMES[2])
    return (h & 0xFFFFFFFF) % lv["size"]


def _level_setup(lv, u):
    s = np.float32(lv["res"])
    p = (u.astype(np.float32) * s).astype(np.float64)
    base = np.clip(np.floor(p), 0, lv["res"] - 1)
    frac = p - base
    return base.astype(np.int64), frac


def encode(lay, params, u):
    """u: [n,3] in [0,1]; returns [n, in_dim] features (zero-padded) and per-level setups."""
    n = len(u)
    feats = np.zeros((n, lay["in_dim"]))
    setups = []
    grid = params[:lay["grid_params"]].reshape(-1, 2)
    for l, lv in enumerate(lay["levels"]):
        base, frac = _level_setup(lv, u)
        table = grid[lv["offset"]: lv["offset"] + lv["size"]]
        acc = np.zeros((n, 2))
        cs = []
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
            w = np.prod(np.where(d[None, :] == 1, frac, 1.0 - frac), axis=1)
            idx = _corner_index(lv, *(base[:, i] + d[i] for i in range(3))).astype(np.int64)
            acc += w[:, None] * table[idx]
            cs.append((idx, w))
        feats[:, 2 * l: 2 * l + 2] = acc
        setups.append(cs)
    return feats, setups


def mlp_weights(lay, params):
    m = lay["mlp"]
    W, IN = lay["width"], lay["in_dim"]
    p = params[lay["grid_params"]:]
    w_in = p[m["w_in"]: m["w_in"] + W * IN].reshape(W, IN)
    w_hid = [p[o: o + W * W].reshape(W, W) for o in m["w_hid"]]
    w_out = p[m["w_out"]: m["w_out"] + W]
    return w_in, w_hid, w_out


def forward(lay, params, u):
    x, setups = encode(lay, params, u)
    w_in, w_hid, w_out = mlp_weights(lay, params)
    acts = []
    h = np.maximum(x @ w_in.T, 0.0)
    acts.append(h)
    for W_ in w_hid:
        h = np.maximum(h @ W_.T, 0.0)
        acts.append(h)
    y = h @ w_out
    return y, {"x": x, "acts": acts, "setups": setups}


def gradients(lay, params, u, t):
    """Gradient of mean((y - t)^2) with respect to every parameter (FP64)."""
    n = len(u)
    y, cache = forward(lay, params, u)
    w_in, w_hid, w_out = mlp_weights(lay, params)
    m = lay["mlp"]
    g = np.zeros_like(params, dtype=np.float64)
    gm = g[lay["grid_params"]:]
    dy = 2.0 * (y - t) / n
    acts = cache["acts"]
    gm[m["w_out"]: m["w_out"] + lay["width"]] = acts[-1].T @ dy
    d = np.outer(dy, w_out) * (acts[-1] > 0)
    for h in range(len(acts) - 1, 0, -1):
        Wh = w_hid[h - 1]
        gm[m["w_hid"][h - 1]: m["w_hid"][h - 1] + Wh.size] = (d.T @ acts[h - 1]).ravel()
        d = (d @ Wh) * (acts[h - 1] > 0)
    gm[m["w_in"]: m["w_in"] + w_in.size] = (d.T @ cache["x"]).ravel()
    dx = d @ w_in
    grid = g[:lay["grid_params"]].reshape(-1, 2)
    for l, lv in enumerate(lay["levels"]):
        for idx, w in cache["setups"][l]:
            np.add.at(grid, lv["offset"] + idx, w[:, None] * dx[:, 2 * l: 2 * l + 2])
    return y, g
