"""CPU oracle of the learned swap-proposal network (test infrastructure only).

Only tests/, the smoke check and bench.py's CPU legs use this module, as the
checker of the CUDA path (brain-match_b200/csrc/bm_mlp.cuh, bm_mlp.cu); it is
never part of the product path.

The reference (brain-match) has no learned component, so this oracle restates
the network's own specification, the one include/bm.h states:

    h1 = relu(W1 x + b1)        x: 128 inputs, W1: 256 x 128
    h2 = relu(W2 h1 + b2)       W2: 256 x 256
    y  = w3 . h2 + b3
    loss = mean_i (y_i - t_i)^2

with the parameters packed as W1, b1, W2, b2, w3, b3.  Two forms:

* ``forward_backward(..., bf16_path=False)`` in float64: the mathematical
  gradient, itself checked against central finite differences in the CPU
  tests (that check pins this oracle);
* ``forward_backward(..., bf16_path=True)``: the same arithmetic with the GPU
  path's bfloat16 roundings (round-to-nearest-even of x, W1, W2, h1, dL/dh2
  and the masked dL/dh1 before each tensor-core product) and float32
  accumulation, so the GPU result agrees to accumulation-order error.

``vertex_features``/``normalise`` restate the feature kernels, pinned by a
hand-computed graph in the CPU tests.
"""
import numpy as np

IN, HID = 128, 256
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("w3", (HID,)), ("b3", (1,))]
COUNT = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + k]).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name]).reshape(-1) for name, _ in SIZES])


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def init_params(seed):
    """He-uniform weights and zero biases (the distribution of bm_mlp_create;
    the generator differs, so tests pass parameters explicitly)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SIZES:
        if name.startswith("b"):
            d[name] = np.zeros(shape)
        else:
            fan_in = shape[-1] if len(shape) > 1 else HID
            lim = np.sqrt(6.0 / fan_in)
            d[name] = rng.uniform(-lim, lim, size=shape)
    return pack(d)


def forward(params, x, bf16_path=True):
    p = unpack(params)
    if bf16_path:
        f = np.float32
        xb = bf16(x)
        h1 = np.maximum(xb @ bf16(p["W1"]).T.astype(f) + p["b1"].astype(f), 0).astype(f)
        h2 = np.maximum(bf16(h1) @ bf16(p["W2"]).T.astype(f) + p["b2"].astype(f), 0).astype(f)
        return (h2 @ p["w3"].astype(f) + f(p["b3"][0])).astype(f)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ p["W1"].T + p["b1"], 0)
    h2 = np.maximum(h1 @ p["W2"].T + p["b2"], 0)
    return h2 @ p["w3"] + p["b3"][0]


def forward_backward(params, x, t, bf16_path=True):
    """Returns (loss, packed gradient) of the mean squared error."""
    p = unpack(params)
    B = len(x)
    if bf16_path:
        f = np.float32
        xb = bf16(x)
        W1b, W2b = bf16(p["W1"]), bf16(p["W2"])
        h1 = np.maximum(xb @ W1b.T + p["b1"].astype(f), 0).astype(f)
        h1b = bf16(h1)
        h2 = np.maximum(h1b @ W2b.T + p["b2"].astype(f), 0).astype(f)
        w3 = p["w3"].astype(f)
        y = (h2 @ w3 + f(p["b3"][0])).astype(f)
        r = (y - np.asarray(t, f)).astype(f)
        loss = float(np.mean(r.astype(np.float64) ** 2))
        dy = (2.0 * r / B).astype(f)
        g = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
        dh2b = bf16(np.where(h2 > 0, dy[:, None] * w3[None, :], 0).astype(f))
        g["W2"] = dh2b.T @ h1b
        g["b2"] = dh2b.sum(0)
        dh1 = (dh2b @ W2b).astype(f)
        dh1m = np.where(h1 > 0, dh1, 0).astype(f)
        g["b1"] = dh1m.sum(0)
        g["W1"] = bf16(dh1m).T @ xb
        return loss, pack(g).astype(np.float32)
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    z1 = x @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0)
    y = h2 @ p["w3"] + p["b3"][0]
    r = y - t
    loss = float(np.mean(r ** 2))
    dy = 2.0 * r / B
    g = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
    dz2 = np.where(z2 > 0, dy[:, None] * p["w3"][None, :], 0)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = np.where(z1 > 0, dz2 @ p["W2"], 0)
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return loss, pack(g)


def finite_difference(params, x, t, idx, eps=1e-6):
    """Central differences of the float64 loss in the coordinates idx."""
    params = np.asarray(params, np.float64)
    out = np.zeros(len(idx))
    for k, i in enumerate(idx):
        pp, pm = params.copy(), params.copy()
        pp[i] += eps
        pm[i] -= eps
        out[k] = (forward_backward(pp, x, t, False)[0] - forward_backward(pm, x, t, False)[0]) / (2 * eps)
    return out


# ---- features (the network's inputs), restated from the feature kernels ----
def vertex_features(n, src1, dst1, w1, src2, dst2, w2, mapping):
    """Per-vertex features F1 (G1 vertices) and F2 (G2 vertices), 32 floats each.

    Ids are 1-based as in the CSV formats; G2 parallel edges keep the last
    weight, G1 parallel edges all count, zero weights are dropped, G1
    self-loops sit apart (feature 8) while G2 self-loops stay in G2's lists.
    mapping[a] is the G2 image of G1 vertex a (1-based, length n+1).  Feature
    columns: 0/1 out/in degree, 2/3 out/in weight sums, 4/5 2-hop out/in
    counts, 6/7 max out/in weight, 8 self-loop weight (G1 only), 9 the current
    overlap contribution (G2: of the G1 vertex mapped onto it), 10 that
    contribution over (incident weight + 1); every column but 10 through
    log1p.  The network sees these after ``normalise``.
    """
    def lists(src, dst, w, dedupe):
        src = np.asarray(src, np.int64) - 1
        dst = np.asarray(dst, np.int64) - 1
        w = np.asarray(w, np.int64)
        if dedupe:
            last = {}
            for s, d, x in zip(src, dst, w):
                last[(s, d)] = x
            return [(s, d, x) for (s, d), x in last.items() if x > 0]
        return [(s, d, x) for s, d, x in zip(src, dst, w) if x > 0]

    g1 = lists(src1, dst1, w1, False)
    g2 = lists(src2, dst2, w2, True)
    self1 = np.zeros(n)
    g1e = []
    for s, d, x in g1:
        if s == d:
            self1[s] += x
        else:
            g1e.append((s, d, x))
    p = np.asarray(mapping, np.int64)[1:] - 1

    def static(edges):
        F = np.zeros((n, 32))
        dego, degi = np.zeros(n), np.zeros(n)
        for s, d, x in edges:
            dego[s] += 1
            degi[d] += 1
        wo, wi, mo, mi, h2o, h2i = (np.zeros(n) for _ in range(6))
        for s, d, x in edges:
            wo[s] += x
            mo[s] = max(mo[s], x)
            h2o[s] += dego[d]
            wi[d] += x
            mi[d] = max(mi[d], x)
            h2i[d] += degi[s]
        for c, v in enumerate([dego, degi, wo, wi, h2o, h2i, mo, mi]):
            F[:, c] = np.log1p(v)
        return F

    F1 = static(g1e)
    F1[:, 8] = np.log1p(self1)
    F2 = static(g2)
    W2 = {(s, d): x for s, d, x in g2}
    contrib = np.zeros(n)
    for s, d, x in g1:  # every G1 entry, parallel and self-loop entries included
        m = min(x, W2.get((p[s], p[d]), 0))
        contrib[s] += m
        if s != d:
            contrib[d] += m
    pinv = np.full(n, -1)
    pinv[p] = np.arange(n)
    tot1 = np.expm1(F1[:, 2]) + np.expm1(F1[:, 3])
    F1[:, 9] = np.log1p(contrib)
    F1[:, 10] = contrib / (tot1 + 1)
    c2 = np.where(pinv >= 0, contrib[np.maximum(pinv, 0)], 0)
    tot2 = np.expm1(F2[:, 2]) + np.expm1(F2[:, 3])
    F2[:, 9] = np.log1p(c2)
    F2[:, 10] = c2 / (tot2 + 1)
    return F1.astype(np.float32), F2.astype(np.float32)


def normalise(F1, F2):
    """Column z-scores over the vertices, as the feature kernels apply them:
    (F - mean) / std with the population std, 0 for a constant column
    (std <= 1e-6)."""
    out = []
    for F in (F1, F2):
        F = np.asarray(F, np.float64)
        mu = F.mean(0)
        sd = np.sqrt(np.maximum((F * F).mean(0) - mu * mu, 0))
        scale = np.where(sd > 1e-6, 1.0 / np.where(sd > 1e-6, sd, 1.0), 0.0)
        out.append(((F - mu) * scale).astype(np.float32))
    return out[0], out[1]


def pair_inputs(F1, F2, mapping, a, b):
    """Network inputs [F1 a, F1 b, F2 p(a), F2 p(b)] of 0-based pairs (a, b)."""
    p = np.asarray(mapping, np.int64)[1:] - 1
    a = np.asarray(a)
    b = np.asarray(b)
    return np.concatenate([F1[a], F1[b], F2[p[a]], F2[p[b]]], axis=1).astype(np.float32)
