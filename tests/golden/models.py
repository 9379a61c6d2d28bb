"""Small test-only models that exercise operators the benchmark workloads do not
(cos, neg, sub of two nodes, reverse-sub, nn.Linear with bias, slices, scalar gathers,
division by a constant, concatenation of several rows), and relaxations that are undefined on
some boxes (log of an interval reaching 0, and sin / exp / square of the resulting unbounded
interval)."""
import torch

F64 = torch.float64


class MixedOps(torch.nn.Module):
    def __init__(self, seed=7):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.lin = torch.nn.Linear(6, 4).to(F64)
        with torch.no_grad():
            self.lin.weight.copy_(torch.randn(4, 6, generator=g, dtype=F64))
            self.lin.bias.copy_(torch.randn(4, generator=g, dtype=F64))
        self.register_buffer("c", torch.randn(4, generator=g, dtype=F64))
        self.box = (-1.5, 1.5)

    def forward(self, x):
        y = self.lin(x)
        z = (y ** 2 + torch.cos(x[:, 1:5]) - 2.0 * y + torch.square(y) + y / 4.0
             - (3.0 - y) + x[:, 2:3] + torch.exp(-0.5 * y) + self.c * torch.sin(y))
        w = torch.log(2.5 + x[:, 0:4] * x[:, 2:6]) - x[:, 3:7 - 3] * y
        return torch.cat([z.sum(1, keepdim=True), (x[:, 0] * 5.0).unsqueeze(1),
                          w.sum(1, keepdim=True), (x[:, 4] - x[:, 5] * x[:, 1]).unsqueeze(1)], 1)


class SinWide(torch.nn.Module):
    """sin/cos on wide and shifted intervals (non-S-shaped branch, table lookups)."""

    def __init__(self, seed=11):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.register_buffer("w", torch.rand(5, generator=g, dtype=F64) * 6 + 0.5)
        self.register_buffer("s", torch.randn(5, generator=g, dtype=F64) * 3)
        self.box = (-3.0, 3.0)

    def forward(self, x):
        a = torch.sin(self.w * x + self.s)
        b = torch.cos(self.w * x - self.s)
        return torch.cat([(a + b).sum(1, keepdim=True), (a * b).sum(1, keepdim=True)], 1)


class DirectOps(torch.nn.Module):
    """Only operators the reference's direct program emitter accepts (nn.Linear with bias, cos,
    neg, sub, slices, gathers, unsqueeze, pow 2, exp, log, concatenation)."""

    def __init__(self, seed=5):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.lin = torch.nn.Linear(6, 3).to(F64)
        with torch.no_grad():
            self.lin.weight.copy_(torch.randn(3, 6, generator=g, dtype=F64))
            self.lin.bias.copy_(torch.randn(3, generator=g, dtype=F64))
        self.register_buffer("idx", torch.tensor([4, 0, 2]))
        self.box = (-1.0, 1.0)

    def forward(self, x):
        y = self.lin(x)
        z = torch.cos(x[:, 1:4]) - y * x[:, self.idx] + torch.exp(-y) + (y ** 2)
        w = torch.log(x[:, 0:3] * x[:, 3:6] + 2.0)
        return torch.cat([z.sum(1, keepdim=True), (-x[:, 5]).unsqueeze(1), w.sum(1, keepdim=True)], 1)


class PowOps(torch.nn.Module):
    """Odd, even and fractional powers (BoundPow): x**3, x**4, x**5 and (x + 2)**1.5, (x + 2)**0.5."""

    def __init__(self, seed=9):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        for name, k in (("a", 4), ("b", 4), ("c", 4), ("d", 4)):
            self.register_buffer(name, torch.randn(k, generator=g, dtype=F64))
        self.box = (-1.2, 1.5)

    def forward(self, x):
        t3 = (x[:, 0:4] ** 3 * self.a).sum(1, keepdim=True)
        t4 = (x[:, 1:5] ** 4 * self.b).sum(1, keepdim=True)
        z = x[:, 2:6] + 2.0
        t15 = (z ** 1.5 * self.c).sum(1, keepdim=True)
        t05 = (z ** 0.5 * self.d).sum(1, keepdim=True)
        return torch.cat([t3 + t4, t15 - t05, (x[:, 5] ** 5).unsqueeze(1)], 1)


class UndefOps(torch.nn.Module):
    """log(x + 0.6) on x in [-1, 1]: its relaxation is undefined on boxes whose interval reaches
    0 (the log's interval is then unbounded below), and so are those of sin, exp and the square of
    that log. Rows: -c log(.) (upper side used), sin(log(.)), exp(log(.)) plus a bilinear, the
    square of the log, and +c log(.) (lower side used)."""

    def __init__(self, seed=13):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.register_buffer("c", torch.rand(3, generator=g, dtype=F64) + 0.5)
        self.register_buffer("d", torch.randn(3, generator=g, dtype=F64))
        self.box = (-1.0, 1.0)

    def forward(self, x):
        L = torch.log(x[:, 0:3] + 0.6)
        f0 = (-self.c * L).sum(1, keepdim=True) + (x[:, 3] * x[:, 4]).unsqueeze(1)
        f1 = (self.d * torch.sin(L)).sum(1, keepdim=True) + x[:, 5:6]
        f2 = torch.exp(L).sum(1, keepdim=True) - (x[:, 0] * x[:, 1]).unsqueeze(1)
        f3 = (L ** 2).sum(1, keepdim=True)
        f4 = (self.c * L).sum(1, keepdim=True)
        return torch.cat([f0, f1, f2, f3, f4], 1)


MODELS = {"mixed_ops": (MixedOps, 6), "sin_wide": (SinWide, 5), "direct_ops": (DirectOps, 6), "pow_ops": (PowOps, 6),
          "undef_ops": (UndefOps, 6)}
