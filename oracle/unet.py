"""TEST INFRASTRUCTURE: the denoiser oracle, a numpy FP64 restatement of the
card's U-Net (mb3d-rs_b200/csrc/dn.cu) for the gradient checks.

The reference renderer has no network of its own (it calls Open Image
Denoise, src/oidn.rs:170-180), so this oracle restates the network the
card defines: 19 3x3 convolutions (zero padding), ReLU after all but the
last, 2x2 max pooling (the first maximum of (0,0) (0,1) (1,0) (1,1) takes
the gradient), nearest 2x upsampling, skip concatenation [upsampled, skip],
channels 32/48/64/80/96, 16 input and 16 output channels (3 used), the
parameters in the card's flat layout (per layer [cout][3][3][cin] weights,
then cout biases), the input log(1 + radiance) | albedo | normal |
depth * scale | zeros, an L1 loss in log space averaged over the valid
pixels' three channels.
"""
import numpy as np

CH = [32, 48, 64, 80, 96]
IN_C = OUT_C = 16


def layers():
    """(cin, cout, relu) of the 19 convolutions in the card's order."""
    L = []
    prev = IN_C
    for l in range(4):
        L += [(prev, CH[l], True), (CH[l], CH[l], True)]
        prev = CH[l]
    L += [(CH[3], CH[4], True), (CH[4], CH[4], True)]
    for l in range(3, -1, -1):
        L += [(CH[l + 1] + CH[l], CH[l], True), (CH[l], CH[l], True)]
    L.append((CH[0], OUT_C, False))
    return L


def unpack(params):
    """[(W (cout, 9, cin), b (cout,))] views of the flat parameters."""
    out, o = [], 0
    for cin, cout, _ in layers():
        w = params[o:o + cout * 9 * cin].reshape(cout, 9, cin)
        o += cout * 9 * cin
        b = params[o:o + cout]
        o += cout
        out.append((w, b))
    assert o == params.size
    return out


def bf16(a):
    """Round to bfloat16 (nearest even), kept in float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def conv(x, w, b):
    """y[n,y,x,co] = sum_tap,ci x[n, y+dy-1, x+dx-1, ci] w[co, tap, ci] + b."""
    n, h, ww, cin = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((n, h, ww, w.shape[0]))
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        y += xp[:, dy:dy + h, dx:dx + ww, :] @ w[:, tap, :].T
    return y + b


def conv_bwd(x, w, dz):
    """(dx, dw, db) of conv for the output gradient dz."""
    n, h, ww, cin = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    dz2 = dz.reshape(-1, dz.shape[-1])
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        dxp[:, dy:dy + h, dx:dx + ww, :] += dz @ w[:, tap, :]
        dw[:, tap, :] = dz2.T @ xp[:, dy:dy + h, dx:dx + ww, :].reshape(-1, cin)
    return dxp[:, 1:-1, 1:-1, :], dw, dz2.sum(axis=0)


def pool(x):
    n, h, w, c = x.shape
    q = [x[:, 0::2, 0::2], x[:, 0::2, 1::2], x[:, 1::2, 0::2], x[:, 1::2, 1::2]]
    return np.maximum(np.maximum(q[0], q[1]), np.maximum(q[2], q[3]))


def pool_bwd(x, dy):
    q = [x[:, 0::2, 0::2], x[:, 0::2, 1::2], x[:, 1::2, 0::2], x[:, 1::2, 1::2]]
    best, arg = q[0].copy(), np.zeros(q[0].shape, np.int64)
    for j in range(1, 4):
        m = q[j] > best
        best = np.where(m, q[j], best)
        arg = np.where(m, j, arg)
    dx = np.zeros_like(x)
    for j, (sy, sx) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        dx[:, sy::2, sx::2] += np.where(arg == j, dy, 0.0)
    return dx


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def up_bwd(dy):
    return dy[:, 0::2, 0::2] + dy[:, 0::2, 1::2] + dy[:, 1::2, 0::2] + dy[:, 1::2, 1::2]


def pack_input(rad, alb, nrm, dep, depth_scale):
    n, h, w, _ = rad.shape
    x = np.zeros((n, h, w, IN_C))
    x[..., 0:3] = np.log1p(np.maximum(rad, 0.0))
    if alb is not None:
        x[..., 3:6] = alb
    if nrm is not None:
        x[..., 6:9] = nrm
    if dep is not None:
        x[..., 9] = dep * depth_scale
    return x


def forward(params, x):
    """The prediction (log space, 16 channels) and the values backward needs."""
    P = unpack(np.asarray(params, np.float64))
    relu = lambda v: np.maximum(v, 0.0)
    c = {"x0": x}
    inp = x
    k = 0
    for l in range(4):
        ea = relu(conv(inp, *P[k]))
        skip = relu(conv(ea, *P[k + 1]))
        c[f"ea{l}"], c[f"skip{l}"] = ea, skip
        inp = pool(skip)
        c[f"pool{l + 1}"] = inp
        k += 2
    ba = relu(conv(inp, *P[8]))
    bb = relu(conv(ba, *P[9]))
    c["ba"], c["bb"] = ba, bb
    low = bb
    k = 10
    for l in range(3, -1, -1):
        cat = np.concatenate([up(low), c[f"skip{l}"]], axis=-1)
        da = relu(conv(cat, *P[k]))
        db = relu(conv(da, *P[k + 1]))
        c[f"cat{l}"], c[f"da{l}"], c[f"db{l}"] = cat, da, db
        low = db
        k += 2
    pred = conv(low, *P[18])
    return pred, c


def l1_loss(pred, target):
    """The loss and its gradient with respect to pred."""
    e = pred[..., :3] - np.log1p(np.maximum(target, 0.0))
    cnt = e.size
    d = np.zeros_like(pred)
    d[..., :3] = np.sign(e) / cnt
    return np.abs(e).sum() / cnt, d


def tone_mse_loss(pred, target, display=False):
    """The squared error of x / (1 + x) (prediction: log(1 + x), its tone
    1 - exp(-pred), pred taken as -30 below -30) and its gradient with
    respect to pred; with display, plus
    the squared error of x clamped to 0..1, its gradient passed through the
    clamp wherever the clamped colours differ (exp(pred) capped at 2)."""
    p = pred[..., :3]
    q = np.exp(-np.maximum(p, -30.0))
    y = np.maximum(target, 0.0)
    e = (1.0 - q) - y / (1.0 + y)
    cnt = e.size
    loss = (e * e).sum()
    g = 2.0 * e * q
    if display:
        ed = np.clip(np.expm1(p), 0.0, 1.0) - np.minimum(y, 1.0)
        loss += (ed * ed).sum()
        g += 2.0 * ed * np.exp(np.minimum(p, np.log(2.0)))
    d = np.zeros_like(pred)
    d[..., :3] = g / cnt
    return loss / cnt, d


def backward(params, c, dpred):
    """The gradient of the loss with respect to every parameter (flat)."""
    P = unpack(np.asarray(params, np.float64))
    G = [None] * 19
    dx, dw, db = conv_bwd(c["db0"], P[18][0], dpred)
    G[18] = (dw, db)
    gdb = dx
    gskip = {}
    for i, l in enumerate(range(0, 4)):
        k = 10 + (3 - l) * 2
        gdb = gdb * (c[f"db{l}"] > 0)
        gda, dw, db = conv_bwd(c[f"da{l}"], P[k + 1][0], gdb)
        G[k + 1] = (dw, db)
        gda = gda * (c[f"da{l}"] > 0)
        gcat, dw, db = conv_bwd(c[f"cat{l}"], P[k][0], gda)
        G[k] = (dw, db)
        nu = CH[l + 1]
        gskip[l] = gcat[..., nu:]
        gdb = up_bwd(gcat[..., :nu])
    gbb = gdb * (c["bb"] > 0)
    gba, dw, db = conv_bwd(c["ba"], P[9][0], gbb)
    G[9] = (dw, db)
    gba = gba * (c["ba"] > 0)
    gpool, dw, db = conv_bwd(c["pool4"], P[8][0], gba)
    G[8] = (dw, db)
    for l in range(3, -1, -1):
        g = gskip[l] + pool_bwd(c[f"skip{l}"], gpool)
        g = g * (c[f"skip{l}"] > 0)
        gea, dw, db = conv_bwd(c[f"ea{l}"], P[2 * l + 1][0], g)
        G[2 * l + 1] = (dw, db)
        gea = gea * (c[f"ea{l}"] > 0)
        x = c["x0"] if l == 0 else c[f"pool{l}"]
        gpool, dw, db = conv_bwd(x, P[2 * l][0], gea)
        G[2 * l] = (dw, db)
    return np.concatenate([np.concatenate([dw.ravel(), db.ravel()]) for dw, db in G])
