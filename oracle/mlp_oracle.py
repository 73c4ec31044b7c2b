"""CPU oracle of the learned pruner's network (test infrastructure only).

A plain-numpy FP64 restatement of the MLP that tsr_b200/csrc/mlp.cu trains
and evaluates: 10 -> 64 -> 64 -> 2 with ReLU, parameters flattened as
W1[10][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2] (W[in][out]), and
the loss the training kernel sums: binary cross-entropy with logits on both
outputs, rows whose label k is 1 weighted by pos_weight[k].

Only tests/ use it, to check the GPU forward pass, the BF16 inference and the
GPU gradients.  There is no counterpart in the reference (the pruner is new).
"""
import numpy as np

NF, NH, NO = 10, 64, 2
SHAPES = [("W1", (NF, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NO)), ("b3", (NO,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], np.float64).ravel() for name, _ in SHAPES])


def init(seed=0):
    """He-style initialisation used by the trainer."""
    rng = np.random.default_rng(seed)
    return pack({"W1": rng.normal(0, np.sqrt(2.0 / NF), (NF, NH)), "b1": np.zeros(NH),
                 "W2": rng.normal(0, np.sqrt(2.0 / NH), (NH, NH)), "b2": np.zeros(NH),
                 "W3": rng.normal(0, np.sqrt(1.0 / NH), (NH, NO)), "b3": np.zeros(NO)})


def forward(theta, x):
    p = unpack(theta)
    x = np.asarray(x, np.float64)
    a1 = x @ p["W1"] + p["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ p["W2"] + p["b2"]
    h2 = np.maximum(a2, 0.0)
    return h2 @ p["W3"] + p["b3"]


def loss_and_grad(theta, x, y, pos_weight=(1.0, 1.0)):
    """Summed weighted BCE-with-logits and its gradient w.r.t. theta."""
    p = unpack(theta)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    a1 = x @ p["W1"] + p["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ p["W2"] + p["b2"]
    h2 = np.maximum(a2, 0.0)
    o = h2 @ p["W3"] + p["b3"]
    w = np.where(y > 0.5, np.asarray(pos_weight, np.float64)[None, :], 1.0)
    loss = np.sum(w * (np.maximum(o, 0.0) - o * y + np.log1p(np.exp(-np.abs(o)))))
    do = w * (1.0 / (1.0 + np.exp(-o)) - y)
    g = {"W3": h2.T @ do, "b3": do.sum(0)}
    d2 = (do @ p["W3"].T) * (a2 > 0)
    g["W2"] = h1.T @ d2
    g["b2"] = d2.sum(0)
    d1 = (d2 @ p["W2"].T) * (a1 > 0)
    g["W1"] = x.T @ d1
    g["b1"] = d1.sum(0)
    return float(loss), pack(g)
