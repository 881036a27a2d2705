"""Fixture-time evaluator for the reference's generated closed forms.

The reference (HyQMOM.jl, ``src/autogen/*.jl``) ships MATLAB-Symbolic-generated
Julia functions (``jacobian6``, ``delta2star3D``, ``rootsR`` ...).  Julia is not
installed here, so this module translates those files, at fixture-generation
time only, into Python callables that evaluate the reference's own expressions
in IEEE double precision.  It is used by ``make_golden.py`` to produce the
committed golden vectors under ``tests/golden/``; nothing else imports it, and
it needs the reference checkout (``HYQMOM_REFERENCE`` env var, default the
read-only mount) to run.  The translated text is never written to disk.

Semantics kept from the reference:
  * ``@fastmath`` real ``sqrt`` of a negative number yields NaN (LLVM fast
    sqrt), so the generated Cardano formulas in ``rootsR``/``rootsR_X_Y`` give
    NaN roots when the cubic has three real roots;
  * ``reshape`` is column-major;
  * ``x^n`` with integer literal n is a plain power.
"""
import math
import os
import re

import numpy as np

REF_ROOT = os.environ.get("HYQMOM_REFERENCE", "/root/reference")


def _fm_sqrt(x):
    if isinstance(x, complex):
        return complex(np.sqrt(x))
    if x != x or x < 0:
        return float("nan")
    return math.sqrt(x)


def _cbrt(x):
    return float(np.cbrt(x))


def _sym_sqrt(A):
    """Principal square root of a symmetric matrix (Julia ``sqrt(::Matrix)``
    takes the Hermitian eigen path for symmetric input)."""
    w, V = np.linalg.eigh(A)
    lam0 = -np.finfo(float).eps * A.shape[0] * np.max(np.abs(w))
    if np.all(w >= lam0):
        w = np.sqrt(np.maximum(w, 0.0))
        return (V * w) @ V.T
    return ((V * np.sqrt(w.astype(complex))) @ V.T).real


_ENV = {
    "sqrt": _fm_sqrt,
    "cbrt": _cbrt,
    "np": np,
    "det": np.linalg.det,
    "real": np.real,
    "msqrt": _sym_sqrt,
}


def _strip(text):
    text = re.sub(r'"""[\s\S]*?"""', "", text)
    out = []
    for line in text.splitlines():
        if "@warn" in line:
            line = line[: line.index("@warn")] + "pass"
        i = line.find("#")
        if i >= 0:
            line = line[:i]
        out.append(line.rstrip())
    return "\n".join(out)


def _split_top(s, sep):
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def _expr(e):
    e = e.strip()
    e = re.sub(r"(\d+(?:\.\d*)?(?:e[+-]?\d+)?)im\b", r"(\1j)", e)
    e = e.replace("^", "**")
    e = re.sub(r"real\(sqrt\((\w+)\)\)", r"msqrt(\1)", e)
    # splat inside array literals
    e = re.sub(r"(\w+)\.\.\.", r"*\1", e)
    # 1-based 2-D indexing A[i,j] on single identifiers
    e = re.sub(r"\b([A-Z]\w*)\[(\d+),(\d+)\]",
               lambda m: f"{m.group(1)}[{int(m.group(2)) - 1},{int(m.group(3)) - 1}]", e)

    def arr(m):
        inner = m.group(1)
        if ";" in inner:
            rows = [r.split() for r in _split_top(inner, ";")]
            return "np.array(\u27e6" + ",".join("\u27e6" + ",".join(r) + "\u27e7" for r in rows) + "\u27e7)"
        return "np.array(\u27e6" + inner + "\u27e7)"

    # innermost bracket literals not preceded by an identifier (indexing)
    prev = None
    while prev != e:
        prev = e
        e = re.sub(r"(?<![\w\]])\[([^\[\]]*)\]", arr, e)
    e = re.sub(r"reshape\((np\.array\(\u27e6[^\u27e7]*\u27e7\)),\s*\(?(\d+),\s*(\d+),\s*(\d+)\)?\)",
               r"np.reshape(\1, (\2,\3,\4), order='F')", e)
    e = re.sub(r"reshape\((np\.array\(\u27e6[^\u27e7]*\u27e7\)),\s*(\d+),\s*(\d+)\)",
               r"np.reshape(\1, (\2,\3), order='F')", e)
    return e.replace("\u27e6", "[").replace("\u27e7", "]")


def translate(name):
    path = os.path.join(REF_ROOT, "src", "autogen", name + ".jl")
    text = _strip(open(path).read())
    m = re.search(r"function\s+(\w+)\(([\s\S]*?)\)\s*\n", text)
    fname, args = m.group(1), m.group(2)
    args = [a.strip() for a in args.replace("\n", " ").split(",") if a.strip()]
    body = text[m.end():]
    # join continuation lines: a statement continues while brackets are open
    stmts, buf, depth = [], "", 0
    for line in body.splitlines():
        s = line.strip()
        if not s:
            continue
        buf = (buf + " " + s) if buf else s
        depth = buf.count("(") + buf.count("[") - buf.count(")") - buf.count("]")
        if depth == 0 and not buf.rstrip().endswith(("+", "-", "*", "/", ",")):
            stmts.extend(_split_top(buf, ";"))
            buf = ""
    py = [f"def {fname}({', '.join(args)}):"]
    indent = 1
    for st in stmts:
        st = st.strip()
        if not st or st == "@fastmath begin":
            continue
        if st == "end":
            indent = max(1, indent - 1) if indent > 1 else indent
            continue
        if st.startswith("if "):
            py.append("    " * indent + "if " + _expr(st[3:]) + ":")
            indent += 1
            continue
        if st.startswith("return "):
            py.append("    " * indent + "return " + _expr(st[7:]))
            continue
        if st == "pass":
            py.append("    " * indent + "pass")
            continue
        lhs, rhs = st.split("=", 1)
        py.append("    " * indent + lhs.strip() + " = " + _expr(rhs))
    src = "\n".join(py)
    env = dict(_ENV)
    exec(compile(src, f"<reference autogen {name}>", "exec"), env)
    return env[fname]


_CACHE = {}


def get(name):
    if name not in _CACHE:
        _CACHE[name] = translate(name)
    return _CACHE[name]
