#!/usr/bin/env python3
"""Generate ws_codelets.cuh: straight-line small DFTs on float2 registers.

Each codelet ``dft<R, INV>(float2 (&v)[R])`` transforms ``v`` in place,
natural order in and out, with sign -1 (forward, MATLAB ``fft``) or +1
(inverse, unnormalised).  Composite sizes use Cooley-Tukey (decimation in time,
input index n = R2*n1 + n2, output index k = k1 + R1*k2) with trivial twiddles
(multiples of pi/4) folded into adds; odd primes use the symmetric-pair form
X[k], X[p-k] = x0 + sum_j a_j cos(2 pi j k / p) -/+ i sum_j b_j sin(2 pi j k / p)
with a_j = x_j + x_{p-j}, b_j = x_j - x_{p-j}.  Constants are computed here in
float64 and written as float literals.

Run:  python gen_codelets.py > ws_codelets.cuh
"""
import math

RADICES = [2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 16]


class Gen:
    def __init__(self):
        self.lines = []
        self.n = 0

    def tmp(self):
        self.n += 1
        return f"t{self.n}"

    def emit(self, s):
        self.lines.append("    " + s)

    # complex value = (re_expr, im_expr) where exprs are variable names or literals
    def cvar(self, re, im):
        a, b = self.tmp(), self.tmp()
        self.emit(f"const float {a} = {re}; const float {b} = {im};")
        return (a, b)

    def add(self, x, y):
        return self.cvar(f"{x[0]} + {y[0]}", f"{x[1]} + {y[1]}")

    def sub(self, x, y):
        return self.cvar(f"{x[0]} - {y[0]}", f"{x[1]} - {y[1]}")

    def mul_twiddle(self, x, m, N, sign):
        """x * exp(sign * 2 pi i m / N)."""
        m %= N
        if m == 0:
            return x
        # exact multiples of pi/4
        if (8 * m) % N == 0:
            e = (8 * m) // N  # angle = sign * e * pi/4
            e = e % 8 if sign > 0 else (-e) % 8
            if e == 0:
                return x
            if e == 2:  # *i
                return self.cvar(f"-{x[1]}", f"{x[0]}")
            if e == 4:
                return self.cvar(f"-{x[0]}", f"-{x[1]}")
            if e == 6:  # *(-i)
                return self.cvar(f"{x[1]}", f"-{x[0]}")
            r = "0.70710678118654752f"
            if e == 1:  # (1+i)/sqrt2
                return self.cvar(f"{r} * ({x[0]} - {x[1]})", f"{r} * ({x[0]} + {x[1]})")
            if e == 3:  # (-1+i)/sqrt2
                return self.cvar(f"-{r} * ({x[0]} + {x[1]})", f"{r} * ({x[0]} - {x[1]})")
            if e == 5:  # (-1-i)/sqrt2
                return self.cvar(f"{r} * ({x[1]} - {x[0]})", f"-{r} * ({x[0]} + {x[1]})")
            if e == 7:  # (1-i)/sqrt2
                return self.cvar(f"{r} * ({x[0]} + {x[1]})", f"{r} * ({x[1]} - {x[0]})")
        ang = sign * 2.0 * math.pi * m / N
        c, s = lit(math.cos(ang)), lit(math.sin(ang))
        return self.cvar(f"fmaf({x[0]}, {c}, -{x[1]} * {s})", f"fmaf({x[0]}, {s}, {x[1]} * {c})")

    def dft(self, xs, sign):
        R = len(xs)
        if R == 1:
            return xs
        if R == 2:
            return [self.add(xs[0], xs[1]), self.sub(xs[0], xs[1])]
        f = first_factor(R)
        if f == R:
            return self.odd_prime(xs, sign)
        R1, R2 = f, R // f
        # inner DFTs of length R1 over n1 for each n2
        inner = []
        for n2 in range(R2):
            col = [xs[R2 * n1 + n2] for n1 in range(R1)]
            d = self.dft(col, sign)
            inner.append([self.mul_twiddle(d[k1], n2 * k1, R, sign) for k1 in range(R1)])
        out = [None] * R
        for k1 in range(R1):
            col = [inner[n2][k1] for n2 in range(R2)]
            d = self.dft(col, sign)
            for k2 in range(R2):
                out[k1 + R1 * k2] = d[k2]
        return out

    def odd_prime(self, xs, p_sign):
        p = len(xs)
        sign = p_sign
        h = (p - 1) // 2
        a = [None] + [self.add(xs[j], xs[p - j]) for j in range(1, h + 1)]
        b = [None] + [self.sub(xs[j], xs[p - j]) for j in range(1, h + 1)]
        s0re = " + ".join([xs[0][0]] + [a[j][0] for j in range(1, h + 1)])
        s0im = " + ".join([xs[0][1]] + [a[j][1] for j in range(1, h + 1)])
        out = [None] * p
        out[0] = self.cvar(s0re, s0im)
        for k in range(1, h + 1):
            tre, tim = xs[0][0], xs[0][1]
            ure, uim = "0.0f", "0.0f"
            first = True
            for j in range(1, h + 1):
                c = lit(math.cos(2 * math.pi * j * k / p))
                s = lit(math.sin(2 * math.pi * j * k / p))
                tre = f"fmaf({a[j][0]}, {c}, {tre})"
                tim = f"fmaf({a[j][1]}, {c}, {tim})"
                if first:
                    ure, uim = f"{b[j][0]} * {s}", f"{b[j][1]} * {s}"
                    first = False
                else:
                    ure = f"fmaf({b[j][0]}, {s}, {ure})"
                    uim = f"fmaf({b[j][1]}, {s}, {uim})"
            T = self.cvar(tre, tim)
            U = self.cvar(ure, uim)
            # forward (sign -1): X_k = T - iU, X_{p-k} = T + iU; inverse swaps
            if sign < 0:
                out[k] = self.cvar(f"{T[0]} + {U[1]}", f"{T[1]} - {U[0]}")
                out[p - k] = self.cvar(f"{T[0]} - {U[1]}", f"{T[1]} + {U[0]}")
            else:
                out[k] = self.cvar(f"{T[0]} - {U[1]}", f"{T[1]} + {U[0]}")
                out[p - k] = self.cvar(f"{T[0]} + {U[1]}", f"{T[1]} - {U[0]}")
        return out


def lit(v):
    if abs(v) < 1e-300:
        v = 0.0
    return f"{v:.17g}f" if "e" not in f"{v:.17g}" else f"{v:.17e}f"


def first_factor(R):
    for f in (4, 2, 3, 5, 7, 11, 13):
        if R % f == 0 and (f != 4 or R != 4):
            return f if R != f else R
    return R


def codelet(R, inverse):
    g = Gen()
    xs = []
    for i in range(R):
        xs.append((f"v[{i}].x", f"v[{i}].y"))
    # copy inputs to locals first (outputs overwrite v)
    loc = [g.cvar(x[0], x[1]) for x in xs]
    sign = 1 if inverse else -1
    if R == 4:
        # radix-4 written directly: 16 real adds, no multiplies
        x0, x1, x2, x3 = loc
        t0 = g.add(x0, x2)
        t1 = g.sub(x0, x2)
        t2 = g.add(x1, x3)
        t3 = g.sub(x1, x3)
        t3r = g.mul_twiddle(t3, 1, 4, sign)  # (x1-x3) * W4^1
        out = [g.add(t0, t2), g.add(t1, t3r), g.sub(t0, t2), g.sub(t1, t3r)]
    else:
        out = g.dft(loc, sign)
    for i, o in enumerate(out):
        g.emit(f"v[{i}] = make_float2({o[0]}, {o[1]});")
    name = "inv" if inverse else "fwd"
    body = "\n".join(g.lines)
    return (f"template <> struct Dft<{R}, {str(inverse).lower()}> {{\n"
            f"  static __host__ __device__ __forceinline__ void run(float2 (&v)[{R}]) {{  // {name}\n{body}\n  }}\n}};\n")


def main():
    out = ["// Generated by gen_codelets.py - do not edit by hand.",
           "// Small in-register DFTs: Dft<R, INV>::run(v) transforms v[0..R) in place,",
           "// natural order, sign -1 (forward) or +1 (inverse, unnormalised).",
           "#pragma once",
           "#include <cuda_runtime.h>",
           "",
           "namespace ws {",
           "",
           "template <int R, bool INV> struct Dft;",
           "template <bool INV> struct Dft<1, INV> { static __host__ __device__ __forceinline__ void run(float2 (&)[1]) {} };",
           ""]
    for R in RADICES:
        for inv in (False, True):
            out.append(codelet(R, inv))
    out.append("constexpr int kNumRadices = %d;" % len(RADICES))
    out.append("constexpr int kRadices[kNumRadices] = {%s};" % ", ".join(map(str, RADICES)))
    out.append("")
    out.append("}  // namespace ws")
    print("\n".join(out))


if __name__ == "__main__":
    main()
