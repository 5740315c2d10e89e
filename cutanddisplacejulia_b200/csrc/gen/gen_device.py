"""Generate ../tde_closed_form.cuh (CUDA device code for the four closed-form
angular-dislocation functions) from the formula table tde_formulas.py.

What the generator does to each function:
  1. keeps every named intermediate of the table as its own value;
  2. splits off every sub-expression that depends only on per-dislocation
     constants (angles, Poisson's ratio, depth) into a setup routine whose
     results are computed once per dislocation and reused for every pair;
  3. replaces x**-k by (1/x)**k with one reciprocal per distinct denominator
     (a reciprocal square root where the denominator is a square root);
  4. runs sympy common-subexpression elimination over all outputs together;
  5. prints straight-line code (integer powers as products): the
     per-dislocation setup in FP64, the per-pair body as a template on its
     arithmetic type R (FP64, or FP32 for far-field pairs), with every literal
     and math function in R.

The result computes the same closed-form mathematics as the reference; only
the association of operations differs.  Usage:
    python gen_device.py            # rewrites ../tde_closed_form.cuh
Requires sympy (development time only).
"""
from __future__ import annotations

import os
import sys

import sympy as sp
from sympy.parsing.sympy_parser import parse_expr

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from tde_formulas import TABLES  # noqa: E402
from sympy.printing.c import C99CodePrinter  # noqa: E402
from sympy.printing.precedence import PRECEDENCE  # noqa: E402

# per-pair inputs of each table (the rest are per-dislocation constants)
PAIR_INPUTS = {
    "ang_dis_disp": ["x", "y", "z"],
    "ang_dis_strain": ["x", "y", "z"],
    "ang_dis_disp_fsc": ["y1", "y2", "y3"],
    "ang_dis_strain_fsc": ["y1", "y2", "y3"],
}


class clampmax(sp.Function):
    """v = clampmax(a, b): `a > b ? b : a` (NaN in a is kept)."""
    nargs = 2


class rcp(sp.Function):
    nargs = 1


class rsq(sp.Function):
    """reciprocal square root"""
    nargs = 1


PI = sp.Symbol("PI", positive=True)


def fix_float_pow(e):
    return e.replace(lambda x: x.is_Pow and x.exp.is_Float and float(x.exp) == int(float(x.exp)),
                     lambda x: sp.Pow(x.base, sp.Integer(int(float(x.exp)))))


def load(fname):
    T = TABLES[fname]
    local = {n: sp.Symbol(n, real=True) for n in T["inputs"]}
    local.update(pi=PI, sqrt=sp.sqrt, log=sp.log, atan=sp.atan)
    defs = []
    for a in T["assigns"]:
        if a[0] == "__clamp__":
            var, val = a[2], a[3]
            new = sp.Symbol(var + "_c", real=True)
            defs.append((new, clampmax(local[var], parse_expr(val, local_dict=local))))
            local[var] = new
            continue
        name, expr = a
        e = fix_float_pow(parse_expr(expr, local_dict=local))
        s = sp.Symbol(name + "_d", real=True)
        defs.append((s, e))
        local[name] = s
    outs = [local[o] for o in T["outputs"]]
    return T, defs, outs


class Hoister:
    def __init__(self, const_syms):
        self.const = set(const_syms)
        self.defs = {}      # expr -> symbol
        self.order = []     # (symbol, expr)

    def is_const(self, e):
        return e.free_symbols <= self.const

    def sym(self, e):
        if e.is_Number or e.is_Symbol:
            return e
        if e not in self.defs:
            s = sp.Symbol("k%d" % len(self.order), real=True)
            self.defs[e] = s
            self.order.append((s, e))
            self.const.add(s)
        return self.defs[e]

    def __call__(self, e):
        if self.is_const(e):
            return self.sym(e)
        if e.is_Mul or e.is_Add:
            cargs = [a for a in e.args if self.is_const(a)]
            vargs = [self(a) for a in e.args if not self.is_const(a)]
            if len(cargs) >= 2 or (len(cargs) == 1 and not (cargs[0].is_Number or cargs[0].is_Symbol)):
                return e.func(self.sym(e.func(*cargs)), *vargs, evaluate=False)
            return e.func(*cargs, *vargs, evaluate=False)
        if e.args:
            return e.func(*[self(a) for a in e.args])
        return e


def reciprocals(exprs, sqrt_defs):
    """Replace x**-k by r**k with r = 1/x (one symbol per distinct x)."""
    table = {}
    order = []

    def rsym(base):
        if base not in table:
            s = sp.Symbol("r%d" % len(order), real=True)
            table[base] = s
            if base in sqrt_defs:          # base = sqrt(arg)
                order.append((s, rsq(sqrt_defs[base])))
            else:
                order.append((s, rcp(base)))
        return table[base]

    def fix(e):
        if e.is_Pow and e.exp.is_Integer and e.exp < 0:
            return sp.Pow(rsym(fix(e.base)), -e.exp, evaluate=False)
        if e.args:
            return e.func(*[fix(a) for a in e.args], evaluate=False) if (e.is_Mul or e.is_Add) else e.func(
                *[fix(a) for a in e.args])
        return e

    return [fix(e) for e in exprs], order


class Printer(C99CodePrinter):
    struct_syms = set()
    pair = False   # printing a per-pair body (literals and functions in R)

    def lit(self, v):
        return ("R(%r)" % v) if self.pair else repr(v)

    def _print_Symbol(self, s):
        if s == PI:
            return "R(M_PI)" if self.pair else "M_PI"
        if s in self.struct_syms:
            return "k." + s.name
        return s.name

    def _print_Float(self, f):
        return self.lit(float(f))

    def _print_Rational(self, r):
        return self.lit(float(r))

    def _print_Integer(self, i):
        return self.lit(float(i))

    def _print_Pow(self, e):
        b, n = e.base, e.exp
        if n == sp.Rational(1, 2):
            return ("cad_sqrt(%s)" if self.pair else "sqrt(%s)") % self._print(b)
        assert n.is_Integer, e
        if n < 0:   # only in per-dislocation setup code
            return "(1.0/%s)" % self._print(sp.Pow(b, -n, evaluate=False))
        bs = self.parenthesize(b, PRECEDENCE["Mul"] + 1)
        n = int(n)
        if n == 1:
            return bs
        return "(" + "*".join([bs] * n) + ")"

    def _print_clampmax(self, e):
        a, b = (self._print(x) for x in e.args)
        return "((%s > %s) ? (%s) : (%s))" % (a, b, b, a)

    def _print_rcp(self, e):
        return "(%s/(%s))" % (self.lit(1.0), self._print(e.args[0]))

    def _print_rsq(self, e):
        return "cad_rsqrt(%s)" % self._print(e.args[0])

    def _print_log(self, e):
        return ("cad_log(%s)" if self.pair else "log(%s)") % self._print(e.args[0])

    def _print_atan(self, e):
        return ("cad_atan(%s)" if self.pair else "atan(%s)") % self._print(e.args[0])


def count_ops(exprs):
    return sum(sp.count_ops(e, visual=False) for e in exprs)


def generate_groups(fname, groups):
    """Hoist per-dislocation constants once for the whole table, then run the
    reciprocal rewrite and CSE separately for every output group."""
    T, defs, outs_all = load(fname)
    pair_in = PAIR_INPUTS[fname]
    const_in = [n for n in T["inputs"] if n not in pair_in]
    const_syms = [sp.Symbol(n, real=True) for n in const_in] + [PI]
    H = Hoister(const_syms)
    pair_defs_all = []
    for s, e in defs:
        if H.is_const(e):
            H.const.add(s)
            H.order.append((s, e))
            H.defs[e] = s
        else:
            pair_defs_all.append((s, H(e)))
    setup_syms = [s for s, _ in H.order]
    setup_rep, setup_red = sp.cse([e for _, e in H.order], symbols=sp.numbered_symbols("c"), optimizations="basic")
    out = []
    for idx in groups:
        outs = outs_all if idx is None else [outs_all[i] for i in idx]
        need = set(outs)
        keep = []
        for s, e in reversed(pair_defs_all):
            if s in need:
                keep.append((s, e))
                need |= e.free_symbols
        pair_defs = list(reversed(keep))
        sqrt_defs = {s: e.args[0] for s, e in pair_defs if e.is_Pow and e.exp == sp.Rational(1, 2)}
        exprs, rorder = reciprocals([e for _, e in pair_defs], sqrt_defs)
        fixed_defs = [(s, e) for (s, _), e in zip(pair_defs, exprs)]
        all_list = [e for _, e in rorder] + [e for _, e in fixed_defs]
        rep, red = sp.cse(all_list, symbols=sp.numbered_symbols("t"), optimizations="basic")
        out.append(dict(T=T, const_in=const_in, pair_in=pair_in, setup_syms=setup_syms, setup_rep=setup_rep,
                        setup_red=setup_red, rorder=rorder, fixed_defs=fixed_defs, rep=rep, red=red,
                        nr=len(rorder), outs=outs, out_idx=idx))
    return out


def topo(stmts, known):
    """Order (symbol, expr) statements so every symbol is defined before use."""
    pending = list(stmts)
    defined = set(known)
    out = []
    while pending:
        progress = False
        rest = []
        for s, e in pending:
            if e.free_symbols <= defined:
                out.append((s, e))
                defined.add(s)
                progress = True
            else:
                rest.append((s, e))
        if not progress:
            raise RuntimeError("cyclic or undefined: %s" % [str(x) for x, _ in rest[:5]])
        pending = rest
    return out


def pair_statements(g):
    nr = g["nr"]
    red = g["red"]
    return list(g["rep"]) + [(s, e) for (s, _), e in zip(g["rorder"], red[:nr])] + \
        [(s, e) for (s, _), e in zip(g["fixed_defs"], red[nr:])]


def used_constants(g):
    stmts = pair_statements(g)
    pair_syms = {s for s, _ in stmts}
    pair_in = {sp.Symbol(n, real=True) for n in g["pair_in"]}
    used = set(g["outs"])
    for _, e in stmts:
        used |= e.free_symbols
    return {x for x in used if x not in pair_syms and x not in pair_in and x != PI}


def emit(fname, groups, P, suffixes):
    L = []
    g0 = groups[0]
    T = g0["T"]
    used_consts = set()
    for g in groups:
        used_consts |= used_constants(g)
    used_consts = sorted(used_consts, key=lambda x: x.name)
    const_in = [sp.Symbol(n, real=True) for n in g0["const_in"]]
    # one constant setup shared by every group
    setup_stmts = list(g0["setup_rep"]) + list(zip(g0["setup_syms"], g0["setup_red"]))
    kname = fname + "_k"
    L.append("// %s: generated from the %s table (reference %s)." % (fname, fname, T["src"]))
    L.append("template <typename T>")
    L.append("struct %s {" % kname)
    for s_ in used_consts:
        L.append("    T %s;" % s_.name)
    L.append("};")
    L.append("")
    args = ", ".join("double %s" % n for n in g0["const_in"])
    L.append("CAD_HD void %s_setup(%s, %s<double>& k)" % (fname, args, kname))
    L.append("{")
    deps = {s_: e_.free_symbols for s_, e_ in setup_stmts}
    live = set()
    stack = list(used_consts)
    while stack:
        x = stack.pop()
        if x in live:
            continue
        live.add(x)
        stack.extend(deps.get(x, ()))
    for s_, e_ in topo([(a, b) for a, b in setup_stmts if a in live], set(const_in) | {PI}):
        L.append("    const double %s = %s;" % (s_.name, P.doprint(e_)))
    for s_ in used_consts:
        L.append("    k.%s = %s;" % (s_.name, s_.name))
    L.append("}")
    L.append("")
    for g, suf in zip(groups, suffixes):
        pargs = ", ".join("R %s" % n for n in g["pair_in"])
        idx = g["out_idx"] or list(range(len(g["outs"])))
        L.append("// outputs %s of %s" % (list(idx), fname))
        L.append("template <typename R>")
        L.append("CAD_HD void %s%s(const %s<R>& k, %s, R* __restrict__ o)" % (
            fname, suf, kname, pargs))
        L.append("{")
        P.struct_syms = set(used_consts)
        P.pair = True
        pair_in = {sp.Symbol(n, real=True) for n in g["pair_in"]}
        for s_, e_ in topo(pair_statements(g), set(used_consts) | pair_in | {PI}):
            L.append("    const R %s = %s;" % (s_.name, P.doprint(e_)))
        for i, o in enumerate(g["outs"]):
            L.append("    o[%d] = %s;" % (i, P.doprint(o)))
        P.struct_syms = set()
        P.pair = False
        L.append("}")
        L.append("")
    return L


# output groups per table: one CSE pass per group (limits live values)
GROUPS = {
    "ang_dis_disp": [None],
    "ang_dis_strain": [None],
    "ang_dis_disp_fsc": [None],
    "ang_dis_strain_fsc": [list(range(0, 6)), list(range(6, 12)), list(range(12, 18))],
}


def main():
    P = Printer()
    out = [
        "// GENERATED by csrc/gen/gen_device.py from csrc/gen/tde_formulas.py -- do not edit.",
        "//",
        "// Device code for the closed-form angular-dislocation terms of the",
        "// triangular dislocation solution (Nikkhoo & Walter 2015):",
        "//   ang_dis_disp, ang_dis_strain            full-space angular dislocation",
        "//   ang_dis_disp_fsc, ang_dis_strain_fsc    half-space free-surface correction",
        "// Each function is split into a per-dislocation setup (constants reused for",
        "// every observation point) and a per-pair body with one reciprocal per",
        "// distinct denominator.  Setup is FP64; the per-pair bodies are templates",
        "// on their arithmetic type R (double, or float for far-field pairs).",
        "// Output order equals the return order of the reference functions.",
        "#pragma once",
        "#include <math.h>",
        "#ifdef __CUDACC__",
        "#include <cuda_runtime.h>",
        "#define CAD_HD __host__ __device__ __forceinline__",
        "#else",
        "#define CAD_HD inline",
        "#endif",
        "",
        "namespace cad {",
        "",
        "#ifndef __CUDACC__",
        "// plain C++ build of the device code (used only to test it on a CPU)",
        "inline double rsqrt(double x) { return 1.0 / sqrt(x); }",
        "inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }",
        "#endif",
        "",
        "// math functions in the pair bodies' arithmetic type",
        "CAD_HD double cad_sqrt(double x) { return sqrt(x); }",
        "CAD_HD float cad_sqrt(float x) { return sqrtf(x); }",
        "CAD_HD double cad_rsqrt(double x) { return rsqrt(x); }",
        "CAD_HD float cad_rsqrt(float x) { return rsqrtf(x); }",
        "CAD_HD double cad_log(double x) { return log(x); }",
        "CAD_HD float cad_log(float x) { return logf(x); }",
        "CAD_HD double cad_atan(double x) { return atan(x); }",
        "CAD_HD float cad_atan(float x) { return atanf(x); }",
        "",
    ]
    stats = {}
    for fname in TABLES:
        spec = GROUPS[fname]
        groups = generate_groups(fname, spec)
        suffixes = [""] if len(spec) == 1 else ["_g%d" % i for i in range(len(spec))]
        out += emit(fname, groups, P, suffixes)
        stats[fname] = (sum(len(g["rep"]) for g in groups), sum(len(g["rorder"]) for g in groups),
                        sum(count_ops([e for _, e in g["rep"]] + list(g["red"])) for g in groups))
    out.append("}  // namespace cad")
    path = os.path.join(HERE, "..", "tde_closed_form.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    for k, v in stats.items():
        print("%-20s cse temps %4d  reciprocals %2d  pair ops ~%d" % (k, *v))


if __name__ == "__main__":
    main()
