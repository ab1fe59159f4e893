"""CPU FP64 restatement of the spike-output surrogate's network (test infrastructure).

Forward: for every linear map but the last, z = h W^T + b, h = SiLU(z) = z sigmoid(z);
the last map gives the logit; the loss is the mean sigmoid cross-entropy.  Backward by
the chain rule.  Parameters use the library's layout (per map: W [out x in] row-major,
then b [out]).  The GPU computes the same in BF16 products with FP32 accumulation, so
tests compare within that precision.
"""
import numpy as np


def _maps(params, dims):
    out, k = [], 0
    for i, o in zip(dims[:-1], dims[1:]):
        W = params[k:k + i * o].reshape(o, i)
        k += i * o
        b = params[k:k + o]
        k += o
        out.append((W, b))
    return out


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def forward(params, dims, x):
    """Logits and the cache of (input, pre-activation) per map."""
    h = np.asarray(x, dtype=np.float64)
    cache = []
    maps = _maps(np.asarray(params, dtype=np.float64), dims)
    for l, (W, b) in enumerate(maps):
        z = h @ W.T + b
        cache.append((h, z))
        h = z * _sigmoid(z) if l + 1 < len(maps) else z
    return h[:, 0], cache


def loss_and_gradients(params, dims, x, y):
    params = np.asarray(params, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    logit, cache = forward(params, dims, x)
    n = len(y)
    loss = np.mean(np.maximum(logit, 0) - logit * y + np.log1p(np.exp(-np.abs(logit))))
    maps = _maps(params, dims)
    grads = []
    dz = ((_sigmoid(logit) - y) / n)[:, None]
    for l in range(len(maps) - 1, -1, -1):
        h, z = cache[l]
        W, _ = maps[l]
        grads.append((dz.T @ h, dz.sum(axis=0)))
        if l == 0:
            break
        dh = dz @ W
        zp = cache[l - 1][1]
        s = _sigmoid(zp)
        dz = dh * (s * (1.0 + zp * (1.0 - s)))
    flat = []
    for dW, db in reversed(grads):
        flat.append(dW.reshape(-1))
        flat.append(db.reshape(-1))
    return loss, np.concatenate(flat)


def predict(params, dims, x):
    logit, _ = forward(params, dims, x)
    return _sigmoid(logit)
