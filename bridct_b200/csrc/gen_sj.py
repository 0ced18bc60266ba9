"""Generator for the Shao-Johnson (SJ) straight-line arithmetic used by the CUDA kernels.

The reference's 1D cores (src/generated/rect_generated.inc:105-9858, src/generated/sj_body.inc)
compute a *scaled* DCT-II of length N: Makhoul's reordering v[n] = x[2n], v[N-1-n] = x[2n+1]
(idx tables, e.g. rect_generated.inc:87), a real split-radix FFT of v in which every
sub-transform is scaled by the Johnson-Frigo factors s(n, k) (leaf* and comb* functions,
tangent twiddles tab*), and a final rotation y[k] = zr - t*zi, y[N-k] = -(zi + t*zr) with
t = -tan(pi k / 2N) (post*_body, rect_generated.inc:89-96).  The output is C[k] / s(4N, k),
where s is `sj_scale` (src/plan.c:40-47); the plan's normalization table undoes the scale.

This module restates that factorization symbolically.  It builds a linear DAG of float
operations (add, sub, neg, multiply by a constant) with hash-consing and algebraic
simplification, so that multiplications by +-1 and additions of 0 vanish exactly as in the
Johnson-Frigo derivation.  The DCT-III (the reference's col_t*/one_t*, "transpose" cores) is
obtained by transposing the DAG, which is how the reference's leafT/combT/post_tbody relate to
leaf/comb/post_body.  The DAG is emitted as CUDA device functions (one thread, registers only)
and is also evaluated in numpy float64 by the self-test in this file.

Scale variants (a restatement of Johnson & Frigo, "A modified split-radix FFT with fewer
arithmetic operations", IEEE TSP 55(1), 2007):
    S  : X_k / s(N, k)        U <- S2_{N/2},  Z, Z' <- S_{N/4}
    S2 : X_k / s(2N, k)       U <- S4_{N/2},  Z, Z' <- S_{N/4}
    S4 : X_k / s(4N, k)       U <- S2_{N/2},  Z, Z' <- S_{N/4}
Every combine multiplies the pair (t Z + t* Z', t Z - t* Z') by t_k = w^k s(N/4,k)/s(N,k),
which is 1 - i tan(2 pi k/N) or cot(2 pi k/N) - i, and then by whatever real ratio of scale
factors the variant needs; the generator computes those ratios in float64 and drops the ones
that equal 1.
"""
from __future__ import annotations

import math
import sys
from typing import Dict, List, Sequence, Tuple

import numpy as np

EPS = 1e-13


def sj_scale(n: int, k: int) -> float:
    """Johnson-Frigo scale factor s(n, k); identical recursion to src/plan.c:40-47."""
    if n <= 4:
        return 1.0
    k %= n // 4
    angle = 2 * math.pi * k / n
    return sj_scale(n // 4, k) * (math.cos(angle) if k <= n // 8 else math.sin(angle))


def variant_scale(variant: str, n: int, k: int) -> float:
    if variant == "1":
        return 1.0
    mult = {"S": 1, "S2": 2, "S4": 4}[variant]
    return sj_scale(mult * n, k)


# ----------------------------------------------------------------------------------------
# Symbolic linear DAG
# ----------------------------------------------------------------------------------------

ZERO = -1


class Graph:
    """Hash-consed DAG of linear float operations.

    Node tuples: ("in", index) | ("add", a, b) | ("sub", a, b) | ("neg", a) | ("mul", a, c).
    The id ZERO stands for an exact 0.0.
    """

    def __init__(self) -> None:
        self.nodes: List[tuple] = []
        self.memo: Dict[tuple, int] = {}

    def _make(self, key: tuple) -> int:
        got = self.memo.get(key)
        if got is not None:
            return got
        self.nodes.append(key)
        idx = len(self.nodes) - 1
        self.memo[key] = idx
        return idx

    def inp(self, i: int) -> int:
        return self._make(("in", i))

    def neg(self, a: int) -> int:
        if a == ZERO:
            return ZERO
        na = self.nodes[a]
        if na[0] == "neg":
            return na[1]
        return self._make(("neg", a))

    def _strip(self, a: int) -> Tuple[int, bool]:
        """Returns (base, negated)."""
        if a != ZERO and self.nodes[a][0] == "neg":
            return self.nodes[a][1], True
        return a, False

    def add(self, a: int, b: int) -> int:
        if a == ZERO:
            return b
        if b == ZERO:
            return a
        ba, na = self._strip(a)
        bb, nb = self._strip(b)
        if na and nb:
            return self.neg(self.add(ba, bb))
        if na:
            return self.sub(b, ba)
        if nb:
            return self.sub(a, bb)
        if a > b:
            a, b = b, a
        return self._make(("add", a, b))

    def sub(self, a: int, b: int) -> int:
        if b == ZERO:
            return a
        if a == ZERO:
            return self.neg(b)
        if a == b:
            return ZERO
        ba, na = self._strip(a)
        bb, nb = self._strip(b)
        if nb:
            return self.add(a, bb)
        if na:
            return self.neg(self.add(ba, b))
        return self._make(("sub", a, b))

    def mul(self, a: int, c: float) -> int:
        if a == ZERO or abs(c) < EPS:
            return ZERO
        if abs(c - 1.0) < EPS:
            return a
        if abs(c + 1.0) < EPS:
            return self.neg(a)
        ba, na = self._strip(a)
        if na:
            return self.mul(ba, -c)
        if c < 0:
            return self.neg(self._make(("mul", a, float(-c))))
        return self._make(("mul", a, float(c)))

    # complex helpers: values are (re, im) tuples of node ids
    def cadd(self, x, y):
        return (self.add(x[0], y[0]), self.add(x[1], y[1]))

    def csub(self, x, y):
        return (self.sub(x[0], y[0]), self.sub(x[1], y[1]))

    def cmulc(self, x, c: complex):
        """x * c for a constant complex c."""
        cr, ci = c.real, c.imag
        re = self.sub(self.mul(x[0], cr), self.mul(x[1], ci))
        im = self.add(self.mul(x[0], ci), self.mul(x[1], cr))
        return (re, im)

    def cscale(self, x, r: float):
        return (self.mul(x[0], r), self.mul(x[1], r))

    def conj(self, x):
        return (x[0], self.neg(x[1]))

    def times_minus_i(self, x):
        return (x[1], self.neg(x[0]))

    def times_i(self, x):
        return (self.neg(x[1]), x[0])

    # numeric evaluation (float64 or complex) for self-tests
    def evaluate(self, outputs: Sequence[int], inputs: np.ndarray) -> np.ndarray:
        vals: Dict[int, np.ndarray] = {}
        zero = np.zeros_like(inputs[0])

        def ev(i: int):
            if i == ZERO:
                return zero
            got = vals.get(i)
            if got is not None:
                return got
            # iterative post-order to avoid deep recursion
            stack = [i]
            while stack:
                n = stack[-1]
                if n in vals:
                    stack.pop()
                    continue
                node = self.nodes[n]
                deps = [d for d in node[1:3] if isinstance(d, int) and node[0] != "in" and d != ZERO]
                if node[0] == "mul":
                    deps = [node[1]] if node[1] != ZERO else []
                pending = [d for d in deps if d not in vals]
                if pending:
                    stack.extend(pending)
                    continue
                op = node[0]
                if op == "in":
                    v = inputs[node[1]]
                elif op == "add":
                    v = vals.get(node[1], zero) + vals.get(node[2], zero)
                elif op == "sub":
                    v = vals.get(node[1], zero) - vals.get(node[2], zero)
                elif op == "neg":
                    v = -vals[node[1]]
                else:
                    v = vals[node[1]] * node[2]
                vals[n] = v
                stack.pop()
            return vals[i]

        return np.array([ev(o) for o in outputs])

    def live(self, outputs: Sequence[int]) -> List[int]:
        """Node ids reachable from outputs, in topological (creation) order."""
        seen = set()
        stack = [o for o in outputs if o != ZERO]
        while stack:
            n = stack.pop()
            if n in seen:
                continue
            seen.add(n)
            node = self.nodes[n]
            if node[0] in ("add", "sub"):
                stack.extend(d for d in node[1:3] if d != ZERO)
            elif node[0] in ("neg", "mul"):
                stack.append(node[1])
        return sorted(seen)

    def count_ops(self, outputs: Sequence[int]) -> Dict[str, int]:
        c = {"add": 0, "mul": 0, "neg": 0}
        for n in self.live(outputs):
            op = self.nodes[n][0]
            if op in ("add", "sub"):
                c["add"] += 1
            elif op == "mul":
                c["mul"] += 1
            elif op == "neg":
                c["neg"] += 1
        return c


def transpose(g: Graph, outputs: Sequence[int], n_inputs: int, adj_inputs: Sequence[int]) -> List[int]:
    """Transposes the linear map inputs -> outputs of `g`.

    `adj_inputs[j]` is the node (in `g` itself) carrying the adjoint of output j.  Returns
    one node per original input i holding (A^T ybar)_i.  Builds the new nodes in `g`, so the
    result can be chained after other computations (round trips).
    """
    order = g.live(outputs)
    contrib: Dict[int, List[int]] = {}
    for o, a in zip(outputs, adj_inputs):
        if o != ZERO:
            contrib.setdefault(o, []).append(a)
    result = [ZERO] * n_inputs
    for n in reversed(order):
        terms = contrib.pop(n, None)
        if not terms:
            continue
        total = terms[0]
        for t in terms[1:]:
            total = g.add(total, t)
        node = g.nodes[n]
        op = node[0]
        if op == "in":
            result[node[1]] = g.add(result[node[1]], total) if result[node[1]] != ZERO else total
        elif op == "add":
            for d in node[1:3]:
                contrib.setdefault(d, []).append(total)
        elif op == "sub":
            contrib.setdefault(node[1], []).append(total)
            contrib.setdefault(node[2], []).append(g.neg(total))
        elif op == "neg":
            contrib.setdefault(node[1], []).append(g.neg(total))
        elif op == "mul":
            contrib.setdefault(node[1], []).append(g.mul(total, node[2]))
    return result


# ----------------------------------------------------------------------------------------
# Johnson-Frigo scaled split-radix (real input, half spectrum) and (complex input)
# ----------------------------------------------------------------------------------------

SUB_VARIANT = {"S": "S2", "S2": "S4", "S4": "S2", "1": "1"}


def rfft(g: Graph, xs: Sequence[int], variant: str) -> List[tuple]:
    """Half spectrum X_k / scale(k), k = 0..N/2, of a real sequence of length N."""
    n = len(xs)
    if n == 1:
        return [(xs[0], ZERO)]
    if n == 2:
        out = [(g.add(xs[0], xs[1]), ZERO), (g.sub(xs[0], xs[1]), ZERO)]
        return [g.cscale(out[k], 1.0 / variant_scale(variant, n, k)) for k in range(2)]
    u = rfft(g, xs[0::2], SUB_VARIANT[variant])
    zvar = "S" if variant != "1" else "1"
    z = rfft(g, xs[1::4], zvar)
    zp = rfft(g, [xs[(4 * m - 1) % n] for m in range(n // 4)], zvar)
    su = lambda j: variant_scale(SUB_VARIANT[variant], n // 2, j)
    sz = lambda j: variant_scale(zvar, n // 4, j)
    sx = lambda j: variant_scale(variant, n, j)
    out: Dict[int, tuple] = {}
    for k in range(0, n // 8 + 1):
        base = sj_scale(n, k) if variant != "1" else 1.0
        # t_k Z_k and conj(t_k) Z'_k with t_k = w^k s_Z(k) / base
        w = complex(math.cos(2 * math.pi * k / n), -math.sin(2 * math.pi * k / n))
        tk = w * sz(k) / base
        tz = g.cmulc(z[k], tk)
        tzp = g.cmulc(zp[k], tk.conjugate())
        a = g.cadd(tz, tzp)
        b = g.csub(tz, tzp)
        uk = u[k]
        uq = g.conj(u[n // 4 - k])  # U_{k+N/4} = conj(U_{N/4-k})
        sk, sq = su(k), su(n // 4 - k)

        def emit(idx, val):
            if 0 <= idx <= n // 2 and idx not in out:
                out[idx] = val

        # X_k = U_k + base*A
        emit(k, g.cadd(g.cscale(uk, sk / sx(k)), g.cscale(a, base / sx(k))))
        # X_{N/2-k} = conj(U_k - base*A)
        emit(n // 2 - k, g.conj(g.csub(g.cscale(uk, sk / sx(n // 2 - k)), g.cscale(a, base / sx(n // 2 - k)))))
        # X_{k+N/4} = U_{k+N/4} - i base*B
        emit(k + n // 4, g.cadd(g.cscale(uq, sq / sx(k + n // 4)),
                                g.times_minus_i(g.cscale(b, base / sx(k + n // 4)))))
        # X_{N/4-k} = conj(U_{k+N/4} + i base*B)
        emit(n // 4 - k, g.conj(g.cadd(g.cscale(uq, sq / sx(n // 4 - k)),
                                       g.times_i(g.cscale(b, base / sx(n // 4 - k))))))
    return [out[k] for k in range(n // 2 + 1)]


def cfft(g: Graph, zs: Sequence[tuple], variant: str) -> List[tuple]:
    """Full spectrum X_k / scale(k), k = 0..N-1, of a complex sequence of length N."""
    n = len(zs)
    if n == 1:
        return [zs[0]]
    if n == 2:
        out = [g.cadd(zs[0], zs[1]), g.csub(zs[0], zs[1])]
        return [g.cscale(out[k], 1.0 / variant_scale(variant, n, k)) for k in range(2)]
    u = cfft(g, zs[0::2], SUB_VARIANT[variant])
    zvar = "S" if variant != "1" else "1"
    z = cfft(g, zs[1::4], zvar)
    zp = cfft(g, [zs[(4 * m - 1) % n] for m in range(n // 4)], zvar)
    su = lambda j: variant_scale(SUB_VARIANT[variant], n // 2, j)
    sz = lambda j: variant_scale(zvar, n // 4, j)
    sx = lambda j: variant_scale(variant, n, j)
    out: List[tuple] = [None] * n  # type: ignore
    for k in range(n // 4):
        base = sj_scale(n, k) if variant != "1" else 1.0
        w = complex(math.cos(2 * math.pi * k / n), -math.sin(2 * math.pi * k / n))
        tk = w * sz(k) / base
        tkp = w.conjugate() * sz(k) / base
        tz = g.cmulc(z[k], tk)
        tzp = g.cmulc(zp[k], tkp)
        a = g.cadd(tz, tzp)
        b = g.csub(tz, tzp)
        uk, uq = u[k], u[k + n // 4]
        s0, s1 = su(k), su(k + n // 4)
        out[k] = g.cadd(g.cscale(uk, s0 / sx(k)), g.cscale(a, base / sx(k)))
        out[k + n // 2] = g.csub(g.cscale(uk, s0 / sx(k + n // 2)), g.cscale(a, base / sx(k + n // 2)))
        out[k + n // 4] = g.cadd(g.cscale(uq, s1 / sx(k + n // 4)),
                                 g.times_minus_i(g.cscale(b, base / sx(k + n // 4))))
        out[k + 3 * n // 4] = g.cadd(g.cscale(uq, s1 / sx(k + 3 * n // 4)),
                                     g.times_i(g.cscale(b, base / sx(k + 3 * n // 4))))
    return out


# ----------------------------------------------------------------------------------------
# DCT-II core (Makhoul + scaled real FFT + tangent post rotation)
# ----------------------------------------------------------------------------------------

def makhoul_index(n: int, j: int) -> int:
    """x index feeding v[j]: v[j] = x[2j] for j < N/2, v[N-1-j] = x[2j+1]."""
    return 2 * j if j < n // 2 else 2 * (n - 1 - j) + 1


def ortho_scale(n: int, k: int) -> float:
    return math.sqrt((1.0 if k == 0 else 2.0) / n)


def plan_scale(n: int, k: int) -> float:
    """Per-axis factor of the reference's normalization table (src/plan.c:92-99)."""
    return sj_scale(4 * n, k) * ortho_scale(n, k)


def dct2_core(g: Graph, xs: Sequence[int], out_scale=None) -> List[int]:
    """Returns y[k] = out_scale[k] * C[k] / s(4N, k) (C = unnormalized DCT-II).

    With out_scale = None the result is the reference's scaled core (one_f*/col_f*); with
    out_scale[k] = plan_scale(N, k) it is the orthonormal DCT-II.
    """
    n = len(xs)
    v = [xs[makhoul_index(n, j)] for j in range(n)]
    z = rfft(g, v, "S")
    ys = [ZERO] * n
    osc = (lambda k: 1.0) if out_scale is None else out_scale
    for k in range(n // 2 + 1):
        th = math.pi * k / (2 * n)
        s_in = sj_scale(n, k)
        if k == 0:
            ys[0] = g.mul(z[0][0], s_in / sj_scale(4 * n, 0) * osc(0))
            continue
        if k == n // 2:
            # V_{N/2} is real; C[N/2] = cos(pi/4) V_{N/2}
            ys[k] = g.mul(z[k][0], s_in * math.cos(th) / sj_scale(4 * n, k) * osc(k))
            continue
        zr, zi = z[k]
        a = s_in / sj_scale(4 * n, k) * osc(k)
        ys[k] = g.add(g.mul(zr, a * math.cos(th)), g.mul(zi, a * math.sin(th)))
        b = s_in / sj_scale(4 * n, n - k) * osc(n - k)
        ys[n - k] = g.sub(g.mul(zr, b * math.sin(th)), g.mul(zi, b * math.cos(th)))
    return ys


# ----------------------------------------------------------------------------------------
# Emission
# ----------------------------------------------------------------------------------------

def fconst(c: float) -> str:
    f = np.float32(c)
    s = repr(float(f))
    if "e" not in s and "." not in s:
        s += ".0"
    return s + "f"


def emit_function(g: Graph, name: str, in_names: Sequence[str], outputs: Sequence[int],
                  out_names: Sequence[str], signature: str, doc: str = "") -> str:
    """Emits a CUDA __device__ function body computing outputs from inputs."""
    order = g.live(outputs)
    lines = []
    if doc:
        lines.append(f"// {doc}")
    lines.append(f"__device__ __forceinline__ void {name}({signature}) {{")
    name_of: Dict[int, str] = {}
    tmp = 0
    for n in order:
        node = g.nodes[n]
        op = node[0]
        if op == "in":
            name_of[n] = f"i{node[1]}"
            lines.append(f"  const float i{node[1]} = {in_names[node[1]]};")
            continue
        t = f"t{tmp}"
        tmp += 1
        if op == "add":
            expr = f"{name_of[node[1]]} + {name_of[node[2]]}"
        elif op == "sub":
            expr = f"{name_of[node[1]]} - {name_of[node[2]]}"
        elif op == "neg":
            expr = f"-{name_of[node[1]]}"
        else:
            expr = f"{name_of[node[1]]} * {fconst(node[2])}"
        lines.append(f"  const float {t} = {expr};")
        name_of[n] = t
    for o, nm in zip(outputs, out_names):
        lines.append(f"  {nm} = {'0.0f' if o == ZERO else name_of[o]};")
    lines.append("}")
    return "\n".join(lines)


# ----------------------------------------------------------------------------------------
# The generated set
# ----------------------------------------------------------------------------------------

REG_SIZES = (8, 16, 32, 64, 128)    # whole line in one thread's registers
LEAF = 32                           # four-step leaf length for N >= 128
STAGE2_SIZES = (4, 8, 16, 32)       # G = N / LEAF


def build_line_ops(n: int):
    """Orthonormal forward (DCT-II), inverse (DCT-III) and round-trip programs for length n."""
    g = Graph()
    xs = [g.inp(i) for i in range(n)]
    fwd = dct2_core(g, xs, out_scale=lambda k: plan_scale(n, k))
    g_inv = Graph()
    ys = [g_inv.inp(i) for i in range(n)]
    # Inverse = transpose of the orthonormal forward; rebuild forward inside g_inv.
    xs2 = [g_inv.inp(n + i) for i in range(n)]  # dummy inputs (forward graph operands)
    fwd2 = dct2_core(g_inv, xs2, out_scale=lambda k: plan_scale(n, k))
    inv = transpose(g_inv, fwd2, 2 * n, ys)[n:]
    g_rt = Graph()
    xr = [g_rt.inp(i) for i in range(n)]
    f = dct2_core(g_rt, xr, out_scale=lambda k: plan_scale(n, k))
    r = transpose(g_rt, f, n, f)
    return (g, fwd), (g_inv, inv), (g_rt, r)


def build_rfft_leaf(n: int):
    """Four-step stage 1: scaled real FFT of length n; outputs re[0..n/2], im[1..n/2-1]."""
    g = Graph()
    xs = [g.inp(i) for i in range(n)]
    z = rfft(g, xs, "S")
    outs = [z[k][0] for k in range(n // 2 + 1)] + [z[k][1] for k in range(1, n // 2)]
    # transpose: inputs are adjoints of outs
    gt = Graph()
    xs_t = [gt.inp(n + i) for i in range(n)]
    zt = rfft(gt, xs_t, "S")
    outs_t = [zt[k][0] for k in range(n // 2 + 1)] + [zt[k][1] for k in range(1, n // 2)]
    adj = [gt.inp(i) for i in range(len(outs_t))]
    back = transpose(gt, outs_t, 2 * n, adj)[n:]
    return (g, outs), (gt, back)


def build_cfft(n: int):
    """Four-step stage 2: scaled complex FFT of length n (S variant) and its transpose."""
    g = Graph()
    zs = [(g.inp(2 * i), g.inp(2 * i + 1)) for i in range(n)]
    z = cfft(g, zs, "S")
    outs = [c for k in range(n) for c in z[k]]
    gt = Graph()
    zs_t = [(gt.inp(2 * n + 2 * i), gt.inp(2 * n + 2 * i + 1)) for i in range(n)]
    zt = cfft(gt, zs_t, "S")
    outs_t = [c for k in range(n) for c in zt[k]]
    adj = [gt.inp(i) for i in range(2 * n)]
    back = transpose(gt, outs_t, 4 * n, adj)[2 * n:]
    return (g, outs), (gt, back)


def build_cfft_half(n: int, half: int):
    """One radix-2 DIF half of a complex FFT of length n (G = 32 stage-2 columns split across
    two lanes): half 0 gives V(2m), half 1 gives V(2m+1), m = 0..n/2-1, each scaled by
    1/s(n/2, m) (an SJ scaled FFT of length n/2 on the folded inputs)."""
    m = n // 2

    def prog(g, zs):
        if half == 0:
            folded = [g.cadd(zs[b], zs[b + m]) for b in range(m)]
        else:
            folded = [g.cmulc(g.csub(zs[b], zs[b + m]),
                              complex(math.cos(2 * math.pi * b / n), -math.sin(2 * math.pi * b / n)))
                      for b in range(m)]
        z = cfft(g, folded, "S")
        return [c for k in range(m) for c in z[k]]
    g = Graph()
    outs = prog(g, [(g.inp(2 * i), g.inp(2 * i + 1)) for i in range(n)])
    gt = Graph()
    outs_t = prog(gt, [(gt.inp(n + 2 * i), gt.inp(n + 2 * i + 1)) for i in range(n)])
    adj = [gt.inp(i) for i in range(n)]
    back = transpose(gt, outs_t, 3 * n, adj)[n:]
    return (g, outs), (gt, back)


def generate() -> str:
    parts = [
        "// Generated by gen_sj.py: Shao-Johnson scaled split-radix arithmetic (straight line).",
        "// Do not edit by hand; rerun `python gen_sj.py > sj_generated.cuh`.",
        "#pragma once",
        "",
    ]
    for n in REG_SIZES:
        (g, fwd), (gi, inv), (gr, rt) = build_line_ops(n)
        ins = [f"v[{i}]" for i in range(n)]
        outs = [f"v[{i}]" for i in range(n)]
        ins2 = ins + ["0.0f"] * n
        for gg, o, nm, kind, in_names in ((g, fwd, f"sj_line_fwd_{n}", "orthonormal DCT-II", ins),
                                          (gi, inv, f"sj_line_inv_{n}", "orthonormal DCT-III", ins2),
                                          (gr, rt, f"sj_line_rt_{n}", "DCT-III(DCT-II(v))", ins)):
            ops = gg.count_ops(o)
            parts.append(emit_function(gg, nm, in_names, o, outs, "float (&v)[%d]" % n,
                                       f"{kind}, length {n}: {ops['add']} add/sub, {ops['mul']} mul"))
            parts.append("")
    (g, outs), (gt, back) = build_rfft_leaf(LEAF)
    m = len(outs)
    parts.append(emit_function(g, f"sj_rfft_{LEAF}", [f"x[{i}]" for i in range(LEAF)], outs,
                               [f"w[{i}]" for i in range(m)],
                               f"const float (&x)[{LEAF}], float (&w)[{m}]",
                               f"scaled real FFT, length {LEAF}: w = re[0..{LEAF//2}], im[1..{LEAF//2-1}]"))
    parts.append("")
    parts.append(emit_function(gt, f"sj_rfft_{LEAF}_t", [f"w[{i}]" for i in range(m)] + ["0.0f"] * LEAF,
                               back, [f"x[{i}]" for i in range(LEAF)],
                               f"const float (&w)[{m}], float (&x)[{LEAF}]",
                               f"transpose of sj_rfft_{LEAF}"))
    parts.append("")
    for half in (0, 1):
        (g, outs), (gt, back) = build_cfft_half(32, half)
        parts.append(emit_function(g, f"sj_cfft_32_half{half}", [f"z[{i}]" for i in range(64)], outs,
                                   [f"o[{i}]" for i in range(32)], "const float (&z)[64], float (&o)[32]",
                                   f"DIF half {half} of the complex FFT of length 32"))
        parts.append("")
        parts.append(emit_function(gt, f"sj_cfft_32_half{half}_t", [f"o[{i}]" for i in range(32)] + ["0.0f"] * 64,
                                   back, [f"z[{i}]" for i in range(64)], "const float (&o)[32], float (&z)[64]",
                                   f"transpose of sj_cfft_32_half{half}"))
        parts.append("")
    for n in STAGE2_SIZES:
        (g, outs), (gt, back) = build_cfft(n)
        parts.append(emit_function(g, f"sj_cfft_{n}", [f"z[{i}]" for i in range(2 * n)], outs,
                                   [f"z[{i}]" for i in range(2 * n)], f"float (&z)[{2 * n}]",
                                   f"scaled complex FFT (S variant), length {n}, interleaved re/im"))
        parts.append("")
        parts.append(emit_function(gt, f"sj_cfft_{n}_t", [f"z[{i}]" for i in range(2 * n)] + ["0.0f"] * (2 * n),
                                   back, [f"z[{i}]" for i in range(2 * n)], f"float (&z)[{2 * n}]",
                                   f"transpose of sj_cfft_{n}"))
        parts.append("")
    return "\n".join(parts)


# ----------------------------------------------------------------------------------------
# Self-test (float64): python gen_sj.py --check
# ----------------------------------------------------------------------------------------

def _dct_matrix(n: int) -> np.ndarray:
    k = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    return np.cos(np.pi * k * (j + 0.5) / n) * np.sqrt(np.where(k == 0, 1.0, 2.0) / n)


def self_check() -> None:
    rng = np.random.default_rng(5)
    for n in REG_SIZES + (128,):
        g = Graph()
        xs = [g.inp(i) for i in range(n)]
        core = dct2_core(g, xs)
        x = rng.standard_normal((n, 3))
        got = g.evaluate(core, x)
        q = _dct_matrix(n)
        want = (q @ x) / np.array([plan_scale(n, k) for k in range(n)])[:, None]
        err = np.abs(got - want).max()
        ops = g.count_ops(core)
        print(f"core N={n}: err {err:.2e}  ops {ops}")
        assert err < 1e-10
    for n in REG_SIZES:
        (g, fwd), (gi, inv), (gr, rt) = build_line_ops(n)
        x = rng.standard_normal((n, 2))
        q = _dct_matrix(n)
        assert np.abs(g.evaluate(fwd, x) - q @ x).max() < 1e-10
        xi = np.concatenate([x, np.zeros_like(x)])
        assert np.abs(gi.evaluate(inv, xi) - q.T @ x).max() < 1e-10
        assert np.abs(gr.evaluate(rt, x) - x).max() < 1e-10
        print(f"line ops N={n}: fwd {g.count_ops(fwd)} inv {gi.count_ops(inv)} rt {gr.count_ops(rt)}")
    for n in STAGE2_SIZES:
        (g, outs), (gt, back) = build_cfft(n)
        z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        flat = np.stack([z.real, z.imag], 1).reshape(-1, 1)
        got = g.evaluate(outs, flat).reshape(n, 2)
        want = np.fft.fft(z) / np.array([sj_scale(n, k) for k in range(n)])
        assert np.abs(got[:, 0] + 1j * got[:, 1] - want).max() < 1e-10
        # transpose check: <A x, y> == <x, A^T y>
        yv = rng.standard_normal((2 * n, 1))
        ax = got.reshape(-1)
        aty = gt.evaluate(back, np.concatenate([yv, np.zeros((2 * n, 1))]))
        assert abs(ax @ yv[:, 0] - flat[:, 0] @ aty[:, 0]) < 1e-9
        print(f"cfft N={n}: ops {g.count_ops(outs)}")
    for half in (0, 1):
        (g, outs), (gt, back) = build_cfft_half(32, half)
        z = rng.standard_normal(32) + 1j * rng.standard_normal(32)
        flat = np.stack([z.real, z.imag], 1).reshape(-1, 1)
        got = g.evaluate(outs, flat).reshape(16, 2)
        f = np.fft.fft(z)[half::2] / np.array([sj_scale(16, k) for k in range(16)])
        assert np.abs(got[:, 0] + 1j * got[:, 1] - f).max() < 1e-10
        yv = rng.standard_normal((32, 1))
        aty = gt.evaluate(back, np.concatenate([yv, np.zeros((64, 1))]))
        assert abs(got.reshape(-1) @ yv[:, 0] - flat[:, 0] @ aty[:, 0]) < 1e-9
        print(f"cfft32 half {half}: ops {g.count_ops(outs)}")
    (g, outs), (gt, back) = build_rfft_leaf(LEAF)
    x = rng.standard_normal((LEAF, 1))
    got = g.evaluate(outs, x)[:, 0]
    f = np.fft.rfft(x[:, 0]) / np.array([sj_scale(LEAF, k) for k in range(LEAF // 2 + 1)])
    want = np.concatenate([f.real, f.imag[1:-1]])
    assert np.abs(got - want).max() < 1e-10
    yv = rng.standard_normal((len(outs), 1))
    aty = gt.evaluate(back, np.concatenate([yv, np.zeros((LEAF, 1))]))
    assert abs(got @ yv[:, 0] - x[:, 0] @ aty[:, 0]) < 1e-9
    print(f"rfft leaf {LEAF}: ops {g.count_ops(outs)}")
    print("OK")


if __name__ == "__main__":
    sys.setrecursionlimit(100000)
    if "--check" in sys.argv:
        self_check()
    else:
        sys.stdout.write(generate() + "\n")
