"""FP64 NumPy restatement of the warm-start encoder-decoder (test infrastructure).

Only tests import this.  It mirrors wavesim_b200/warmstart.py operation by
operation (same channels-last layout, the same im2col ordering of the 3x3x3
taps ((dz*3 + dy)*3 + dx)*C + c, zero padding 1, 2x2x2 average pooling,
nearest x2 upsampling with channel concat, ReLU) and back-propagates by hand,
so that the GPU forward pass and every layer's weight, bias and input
gradients can be compared with it on small volumes.  The network has no
counterpart in the reference; nothing here pins against it.
"""
import numpy as np


def im2col(x, vol, C):
    b, d, h, w = vol
    xv = x.reshape(b, d, h, w, C)
    xp = np.pad(xv, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    cols = []
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        cols.append(xp[:, dz:dz + d, dy:dy + h, dx:dx + w, :])
    return np.concatenate(cols, axis=-1).reshape(b * d * h * w, 27 * C)


def col2im(dcol, vol, C):
    b, d, h, w = vol
    dc = dcol.reshape(b, d, h, w, 27 * C)
    dxp = np.zeros((b, d + 2, h + 2, w + 2, C))
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        dxp[:, dz:dz + d, dy:dy + h, dx:dx + w, :] += dc[..., t * C:(t + 1) * C]
    return dxp[:, 1:-1, 1:-1, 1:-1, :].reshape(b * d * h * w, C)


def pool(x, vol, C):
    b, d, h, w = vol
    return x.reshape(b, d // 2, 2, h // 2, 2, w // 2, 2, C).mean(axis=(2, 4, 6)).reshape(-1, C)


def pool_grad(g, vol, C):
    b, d, h, w = vol
    gv = g.reshape(b, d // 2, h // 2, w // 2, C) / 8.0
    return np.repeat(np.repeat(np.repeat(gv, 2, 1), 2, 2), 2, 3).reshape(-1, C)


def upcat(a, skip, vol, ca, cs):
    b, d, h, w = vol
    av = a.reshape(b, d // 2, h // 2, w // 2, ca)
    up = np.repeat(np.repeat(np.repeat(av, 2, 1), 2, 2), 2, 3).reshape(-1, ca)
    return np.concatenate([up, skip], axis=1)


def upcat_grad(g, vol, ca, cs):
    b, d, h, w = vol
    ga = g[:, :ca].reshape(b, d // 2, 2, h // 2, 2, w // 2, 2, ca).sum(axis=(2, 4, 6)).reshape(-1, ca)
    return ga, g[:, ca:].copy()


class Net:
    """weights: list of (W [Cout][27 Cin], b [Cout]) in the layer order of WarmStartNet.layers."""

    def __init__(self, weights, widths):
        self.W = [(np.asarray(w, np.float64), np.asarray(b, np.float64)) for w, b in weights]
        self.widths = widths

    def conv(self, i, x, vol, relu=True):
        W, b = self.W[i]
        cin = W.shape[1] // 27
        col = im2col(x, vol, cin)
        y = col @ W.T + b
        return (np.maximum(y, 0) if relu else y), col

    def forward(self, x, vol):
        w1, w2, w3, w4 = self.widths
        b, d, h, w = vol
        v = [vol, (b, d // 2, h // 2, w // 2), (b, d // 4, h // 4, w // 4), (b, d // 8, h // 8, w // 8)]
        a = {"x": x}
        a["e1a"], a["c0"] = self.conv(0, x, v[0])
        a["e1"], a["c1"] = self.conv(1, a["e1a"], v[0])
        a["p1"] = pool(a["e1"], v[0], w1)
        a["e2a"], a["c2"] = self.conv(2, a["p1"], v[1])
        a["e2"], a["c3"] = self.conv(3, a["e2a"], v[1])
        a["p2"] = pool(a["e2"], v[1], w2)
        a["e3a"], a["c4"] = self.conv(4, a["p2"], v[2])
        a["e3"], a["c5"] = self.conv(5, a["e3a"], v[2])
        a["p3"] = pool(a["e3"], v[2], w3)
        a["b4a"], a["c6"] = self.conv(6, a["p3"], v[3])
        a["b4"], a["c7"] = self.conv(7, a["b4a"], v[3])
        a["u3"] = upcat(a["b4"], a["e3"], v[2], w4, w3)
        a["d3a"], a["c8"] = self.conv(8, a["u3"], v[2])
        a["d3"], a["c9"] = self.conv(9, a["d3a"], v[2])
        a["u2"] = upcat(a["d3"], a["e2"], v[1], w3, w2)
        a["d2a"], a["c10"] = self.conv(10, a["u2"], v[1])
        a["d2"], a["c11"] = self.conv(11, a["d2a"], v[1])
        a["u1"] = upcat(a["d2"], a["e1"], v[0], w2, w1)
        a["d1a"], a["c12"] = self.conv(12, a["u1"], v[0])
        a["d1"], a["c13"] = self.conv(13, a["d1a"], v[0])
        out, a["c14"] = self.conv(14, a["d1"], v[0], relu=False)
        return out, a

    def backward(self, a, dout, vol):
        """Returns [(dW, db)] per layer for the gradient dout of the output."""
        w1, w2, w3, w4 = self.widths
        b, d, h, w = vol
        v = [vol, (b, d // 2, h // 2, w // 2), (b, d // 4, h // 4, w // 4), (b, d // 8, h // 8, w // 8)]
        grads = [None] * 15

        def conv_b(i, g, y, vl, relu=True):
            if relu:
                g = g * (y > 0)
            W, _ = self.W[i]
            col = a[f"c{i}"]
            grads[i] = (g.T @ col, g.sum(axis=0))
            return col2im(g @ W, vl, W.shape[1] // 27)

        g = conv_b(14, dout, None, v[0], relu=False)
        g = conv_b(13, g, a["d1"], v[0])
        g = conv_b(12, g, a["d1a"], v[0])
        g_d2, g_e1 = upcat_grad(g, v[0], w2, w1)
        g = conv_b(11, g_d2, a["d2"], v[1])
        g = conv_b(10, g, a["d2a"], v[1])
        g_d3, g_e2 = upcat_grad(g, v[1], w3, w2)
        g = conv_b(9, g_d3, a["d3"], v[2])
        g = conv_b(8, g, a["d3a"], v[2])
        g_b4, g_e3 = upcat_grad(g, v[2], w4, w3)
        g = conv_b(7, g_b4, a["b4"], v[3])
        g = conv_b(6, g, a["b4a"], v[3])
        g = pool_grad(g, v[2], w3) + g_e3
        g = conv_b(5, g, a["e3"], v[2])
        g = conv_b(4, g, a["e3a"], v[2])
        g = pool_grad(g, v[1], w2) + g_e2
        g = conv_b(3, g, a["e2"], v[1])
        g = conv_b(2, g, a["e2a"], v[1])
        g = pool_grad(g, v[0], w1) + g_e1
        g = conv_b(1, g, a["e1"], v[0])
        conv_b(0, g, a["e1a"], v[0])
        return grads
