"""CPU reference of the learned warm-start network (test infrastructure only).

NumPy restatement of gample_b200/csrc/learned.cu: the same 12 3x3 conv
layers (32/64/128/256 channels, skip connections, 2x2 average pooling,
nearest upsampling), ReLU, mean-squared-error loss and backward pass, with the
GPU's BF16 roundings emulated where the GPU rounds (GEMM operands:
activations, pre-activation gradients, weights) and FP64 accumulation
elsewhere. Used to check the GPU forward pass and gradients.
"""
import numpy as np

SPECS = [(2, 32, True), (32, 32, True), (32, 64, True), (64, 64, True), (64, 128, True), (128, 128, True),
         (128, 256, True), (256, 256, True), (384, 128, True), (192, 64, True), (96, 32, True), (32, 1, False)]


def bf16(x):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    x32 = np.ascontiguousarray(x, np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def im2col(x):
    """x (h, w, c) -> (h*w, 9c), column t*c + ch = x[y + t//3 - 1, x + t%3 - 1, ch]."""
    h, w, c = x.shape
    p = np.zeros((h + 2, w + 2, c))
    p[1:-1, 1:-1] = x
    cols = [p[dy:dy + h, dx:dx + w] for dy in range(3) for dx in range(3)]
    return np.concatenate(cols, axis=2).reshape(h * w, 9 * c)


def col2im(g, h, w, c):
    """Adjoint of im2col."""
    g = g.reshape(h, w, 9, c)
    p = np.zeros((h + 2, w + 2, c))
    t = 0
    for dy in range(3):
        for dx in range(3):
            p[dy:dy + h, dx:dx + w] += g[:, :, t]
            t += 1
    return p[1:-1, 1:-1]


def pool(x):
    h, w, c = x.shape
    return 0.25 * x.reshape(h // 2, 2, w // 2, 2, c).sum(axis=(1, 3))


def pool_back(g):
    return 0.25 * np.repeat(np.repeat(g, 2, axis=0), 2, axis=1)


def up(x):
    return np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)


def up_back(g):
    h, w, c = g.shape
    return g.reshape(h // 2, 2, w // 2, 2, c).sum(axis=(1, 3))


class RefNet:
    def __init__(self, weights, biases, round_bf16=True):
        """weights[i]: (cout, kpad) FP32 masters (columns >= 9 cin unused), biases[i]: (cout,).
        round_bf16=False: plain FP64 (for finite-difference checks of this code)."""
        self.r = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
        self.W = [self.r(np.asarray(w, np.float64)[:, :9 * s[0]]) for w, s in zip(weights, SPECS)]
        self.b = [np.asarray(b, np.float64) for b in biases]

    def _conv(self, i, x, last=False):
        y = im2col(x) @ self.W[i].T + self.b[i]
        if SPECS[i][2]:
            y = np.maximum(y, 0.0)
        h, w, _ = x.shape
        y = y.reshape(h, w, -1)
        return y if last else self.r(y)

    def forward(self, inp):
        r = self.r
        a = {0: r(inp)}
        a[1] = self._conv(0, a[0])
        a[2] = self._conv(1, a[1])
        a[3] = r(pool(a[2]))
        a[4] = self._conv(2, a[3])
        a[5] = self._conv(3, a[4])
        a[6] = r(pool(a[5]))
        a[7] = self._conv(4, a[6])
        a[8] = self._conv(5, a[7])
        a[9] = r(pool(a[8]))
        a[10] = self._conv(6, a[9])
        a[11] = self._conv(7, a[10])
        a[12] = np.concatenate([up(a[11]), a[8]], axis=2)
        a[13] = self._conv(8, a[12])
        a[14] = np.concatenate([up(a[13]), a[5]], axis=2)
        a[15] = self._conv(9, a[14])
        a[16] = np.concatenate([up(a[15]), a[2]], axis=2)
        a[17] = self._conv(10, a[16])
        a[18] = self._conv(11, a[17], last=True)
        self.a = a
        return a[18][:, :, 0]

    def loss_grad(self, inp, target):
        out = self.forward(inp)
        n = out.size
        d = out - target
        loss = float(np.mean(d * d))
        a = self.a
        g = {k: np.zeros_like(v) for k, v in a.items()}
        g[18] = (2.0 * d / n)[:, :, None]
        gw, gb = [None] * 12, [None] * 12

        def back(i, xi, yi, need_dx=True):
            y = a[yi]
            gy = g[yi]
            if SPECS[i][2]:
                gy = gy * (y > 0)
            gb[i] = gy.reshape(-1, gy.shape[2]).sum(axis=0)
            gyb = self.r(gy).reshape(-1, gy.shape[2])
            x = a[xi]
            gw[i] = gyb.T @ im2col(x)
            if need_dx:
                h, w, c = x.shape
                g[xi] += col2im(gyb @ self.W[i], h, w, c)

        back(11, 17, 18)
        back(10, 16, 17)
        g[15] += up_back(g[16][:, :, :64])
        g[2] += g[16][:, :, 64:]
        back(9, 14, 15)
        g[13] += up_back(g[14][:, :, :128])
        g[5] += g[14][:, :, 128:]
        back(8, 12, 13)
        g[11] += up_back(g[12][:, :, :256])
        g[8] += g[12][:, :, 256:]
        back(7, 10, 11)
        back(6, 9, 10)
        g[8] += pool_back(g[9])
        back(5, 7, 8)
        back(4, 6, 7)
        g[5] += pool_back(g[6])
        back(3, 4, 5)
        back(2, 3, 4)
        g[2] += pool_back(g[3])
        back(1, 1, 2)
        back(0, 0, 1, need_dx=False)
        return loss, gw, gb
