"""CPU oracle for the learned DROP initializer (TEST INFRASTRUCTURE ONLY: imported by tests/ and
never by the engine).

The reference has no learned component, so there is nothing of the reference's to restate here;
this is an independent numpy statement of the network the engine runs (pct_unet.cu): 3x3x3
convolutions with zero padding, ReLU, 2x2x2 average pooling, nearest x2 upsampling with additive
skips, image = x_0 + hull * output, masked mean-squared-error loss, and the analytic backward pass.

Two modes:
  * quantize=True rounds to bf16 (round to nearest even) exactly where the engine stores bf16:
    the packed input, weights, every activation and every gradient tensor; sums are formed in
    float64 (the engine sums in fp32), so the two agree to accumulation-order differences;
  * quantize=False keeps float64 throughout; tests pin this mode's analytic gradients against
    central finite differences.

Layer table (cin, cout, level, input, upsample, residual) -- the same network as the engine's:
  input -1 = the packed volume, 'pool' = avg-pool of the previous level's encoder output.
"""
from __future__ import annotations

import numpy as np

LAYERS = [
    (16, 16, 0, -1, 0, -1), (16, 16, 0, 0, 0, -1),
    (16, 32, 1, "pool", 0, -1), (32, 32, 1, 2, 0, -1),
    (32, 64, 2, "pool", 0, -1), (64, 64, 2, 4, 0, -1),
    (64, 128, 3, "pool", 0, -1), (128, 128, 3, 6, 0, -1),
    (128, 64, 2, 7, 1, 5), (64, 64, 2, 8, 0, -1),
    (64, 32, 1, 9, 1, 3), (32, 32, 1, 10, 0, -1),
    (32, 16, 0, 11, 1, 1), (16, 16, 0, 12, 0, -1),
    (16, 16, 0, 13, 0, -1),
]
OFFSETS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def bf16(a) -> np.ndarray:
    """Round float32 values to bf16 (nearest, ties to even); result as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(a) -> np.ndarray:
    """bf16 bit patterns (uint16) of float32 values, rounded to nearest even."""
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def param_layout():
    """(weight offset, bias offset) per layer in the flat parameter vector, and its length."""
    offs, o = [], 0
    for cin, cout, *_ in LAYERS:
        offs.append((o, o + cout * 27 * cin))
        o += cout * 27 * cin + cout
    return offs, o


def upsample(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def conv3d(x, w, up=False):
    """sum_{t,ci} w[co,t,ci] x[v + offset_t, ci] with zero padding; x [D,H,W,Cin], w [Cout,27,Cin];
    float64 result [D,H,W,Cout] (at twice x's resolution when up)."""
    if up:
        x = upsample(x)
    D, H, W, C = x.shape
    xp = np.pad(x.astype(np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((D, H, W, w.shape[0]), np.float64)
    for t, (dz, dy, dx) in enumerate(OFFSETS):
        sl = xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]
        out += sl @ w[:, t, :].astype(np.float64).T
    return out


def conv3d_wgrad(x, dz, up=False):
    """dW[co,t,ci] = sum_v dz[v,co] x[v + offset_t, ci] (float64)."""
    if up:
        x = upsample(x)
    D, H, W, C = x.shape
    xp = np.pad(x.astype(np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    g = dz.astype(np.float64).reshape(-1, dz.shape[-1])
    dw = np.zeros((dz.shape[-1], 27, C), np.float64)
    for t, (oz, oy, ox) in enumerate(OFFSETS):
        sl = xp[1 + oz:1 + oz + D, 1 + oy:1 + oy + H, 1 + ox:1 + ox + W].reshape(-1, C)
        dw[:, t, :] = g.T @ sl
    return dw


def conv3d_dgrad(dz, w):
    """Gradient with respect to the (possibly upsampled) input: the convolution of dz with the
    flipped, transposed kernel w'[ci, 26 - t, co] = w[co, t, ci]."""
    wt = np.transpose(w[:, ::-1, :], (2, 1, 0))
    return conv3d(dz, wt)


def avgpool(x):
    D, H, W, C = x.shape
    return x.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).astype(np.float64).mean(axis=(1, 3, 5))


class UNetOracle:
    def __init__(self, params, quantize=True):
        self.params = np.asarray(params, np.float64)
        self.quantize = quantize
        self.offs, n = param_layout()
        assert len(self.params) == n

    def q(self, a):
        return bf16(a).astype(np.float64) if self.quantize else np.asarray(a, np.float64)

    def weight(self, l):
        cin, cout = LAYERS[l][:2]
        o, b = self.offs[l]
        w = self.params[o:b].reshape(cout, 27, cin)
        return self.q(w), self.params[b:b + cout]

    def input_of(self, l):
        src = LAYERS[l][3]
        if src == -1:
            return self.x_in
        if src == "pool":
            return self.pools[LAYERS[l][2]]
        return self.act[src]

    def forward(self, x0, hull, shape):
        """x0 (float32 [V]) and hull (0/1 [V]) in voxel order; shape = (slices, rows, columns)."""
        D, H, W = shape
        self.shape, self.hull = shape, np.asarray(hull).reshape(D, H, W) != 0
        self.x0 = np.asarray(x0, np.float32).reshape(D, H, W).astype(np.float64)
        x = np.zeros((D, H, W, 16))
        x[..., 0] = self.x0
        x[..., 1] = self.hull
        self.x_in = self.q(x)
        self.act, self.pools = {}, {}
        for l, (cin, cout, level, src, up, res) in enumerate(LAYERS):
            if src == "pool":
                self.pools[level] = self.q(avgpool(self.act[2 * (level - 1) + 1]))
            w, b = self.weight(l)
            z = conv3d(self.input_of(l), w, bool(up))
            if self.quantize:
                z = z.astype(np.float32).astype(np.float64)
            z = z + b
            if res >= 0:
                z = z + self.act[res]
            if l == len(LAYERS) - 1:
                self.y = self.x0 + np.where(self.hull, z[..., 0], 0.0)
                return self.y.reshape(-1)
            self.act[l] = self.q(np.maximum(z, 0.0))

    def loss_and_gradients(self, x0, hull, target, shape):
        y = self.forward(x0, hull, shape).reshape(shape)
        t = np.asarray(target, np.float32).reshape(shape).astype(np.float64)
        m = self.hull
        count = max(int(m.sum()), 1)
        d = np.where(m, y - t, 0.0)
        loss = float((d * d).sum() / count)
        grads = np.zeros_like(self.params)
        dz = {}
        g = np.zeros(shape + (16,))
        g[..., 0] = 2.0 * d / count
        dz[len(LAYERS) - 1] = self.q(g)
        skip_of = {res: l for l, (*_, res) in enumerate(LAYERS) if res >= 0}
        for l in range(len(LAYERS) - 1, -1, -1):
            cin, cout, level, src, up, res = LAYERS[l]
            o, b = self.offs[l]
            grads[o:b] = conv3d_wgrad(self.input_of(l), dz[l], bool(up)).reshape(-1)
            grads[b:b + cout] = dz[l].reshape(-1, cout).sum(axis=0)
            if l == 0:
                break
            w, _ = self.weight(l)
            dx = conv3d_dgrad(dz[l], w)
            if self.quantize:
                dx = dx.astype(np.float32).astype(np.float64)
            if up:
                Dc, Hc, Wc = self.act[src].shape[:3]
                s = self.q(dx).reshape(Dc, 2, Hc, 2, Wc, 2, cin).sum(axis=(1, 3, 5))
                dz[src] = self.q(np.where(self.act[src] > 0, s, 0.0))
            elif src == "pool":
                e = 2 * (level - 1) + 1
                dp = self.q(dx)
                fine = upsample(dp) * 0.125 + dz[skip_of[e]]
                dz[e] = self.q(np.where(self.act[e] > 0, fine, 0.0))
            else:
                dz[src] = self.q(np.where(self.act[src] > 0, dx, 0.0))
        return loss, grads
