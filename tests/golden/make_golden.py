"""Generate pfpx_golden.npz from the reference's own generated barrier Jacobians.

The reference's barrier kernel (StiffGIPC/GIPC.cu:3106-4945, NEWF path) takes its
distance derivatives from straight-line code emitted by MATLAB's Symbolic Math Toolbox in
StiffGIPC/GIPC_PDerivative.cuh: pFpx_pp2, pFpx_pe2, pFpx_pt2, pFpx_ee2 (the last column is
d(d/sqrt(dhat))/dx) and pFpx_pppV0V1, pFpx_ppeV0V1, pFpx_peeV0V1 for the mollified pairs
(column 4 is dc/dx, c = |e0 x e1|; column 8 as above).  This script reads those function
bodies from a reference checkout, evaluates their arithmetic verbatim (each `t = expr;`
statement executed in order) at seeded configurations and stores inputs and outputs.
Nothing of the source is stored; the fixture holds numbers only.

Usage: python tests/golden/make_golden.py [path/to/StiffGIPC]   (default /root/reference/StiffGIPC)
"""
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# function -> (number of vertices, reference pair encoding kind used by the oracle)
FUNCS = {
    "pFpx_pp2": 2,
    "pFpx_pe2": 3,
    "pFpx_pt2": 4,
    "pFpx_ee2": 4,
    "pFpx_pppV0V1": 4,
    "pFpx_ppeV0V1": 4,
    "pFpx_peeV0V1": 4,
}


def extract(src, name):
    m = re.search(r"void\s+%s\s*\(\s*double\s+d\s*," % name, src)
    if not m:
        raise KeyError(name)
    start = src.index("{", m.end())
    depth, i = 0, start
    while True:
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[start + 1:i]
        i += 1


def evaluate(body, d, x, shape):
    env = {"sqrt": math.sqrt, "pow": math.pow, "fabs": abs, "d": d}
    names = ["x11", "x12", "x13", "x21", "x22", "x23", "x31", "x32", "x33", "x41", "x42", "x43"]
    for n, v in zip(names, x):
        env[n] = v
    out = np.zeros(shape)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    for stmt in body.split(";"):
        s = stmt.strip()
        if not s or s.startswith("double "):
            continue
        lhs, rhs = s.split("=", 1)
        lhs = lhs.strip()
        rhs = " ".join(rhs.split())
        op = lhs[-1] if lhs[-1] in "+-*/" else None   # compound assignment, e.g. `t78 *= t76`
        if op:
            lhs = lhs[:-1].strip()
            rhs = "(%s) %s (%s)" % (lhs, op, rhs)
        val = eval(rhs, {"__builtins__": {}}, env)  # noqa: S307 - arithmetic of a trusted local checkout
        m = re.fullmatch(r"result\[(\d+)\](?:\[(\d+)\])?", lhs)
        if m:
            if m.group(2) is None:
                out[int(m.group(1))] = val
            else:
                out[int(m.group(1)), int(m.group(2))] = val
        else:
            env[lhs] = val
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/StiffGIPC"
    src = open(os.path.join(ref, "GIPC_PDerivative.cuh")).read()
    rng = np.random.default_rng(20240601)
    data = {}
    for name, nv in FUNCS.items():
        body = extract(src, name)
        xs, ds, outs = [], [], []
        for _ in range(8):
            base = rng.uniform(-0.05, 0.05, 3)
            X = base + rng.uniform(-2e-3, 2e-3, (4, 3))
            if name in ("pFpx_pppV0V1", "pFpx_ppeV0V1", "pFpx_peeV0V1"):
                # nearly parallel edges, the regime the mollifier covers
                e = rng.normal(size=3)
                e /= np.linalg.norm(e)
                X[1] = X[0] + 4e-3 * e + rng.uniform(-1e-5, 1e-5, 3)
                X[3] = X[2] + 4e-3 * e + rng.uniform(-1e-5, 1e-5, 3)
            d = math.sqrt(1e-6)
            shape = (6,) if name == "pFpx_pp2" else (3 * nv, 9) if name == "pFpx_pe2" else (12, 9)
            out = evaluate(body, d, X.reshape(-1), shape)
            xs.append(X)
            ds.append(d)
            outs.append(out)
        data[name + "_x"] = np.array(xs)
        data[name + "_d"] = np.array(ds)
        data[name + "_out"] = np.array(outs)
    np.savez(os.path.join(HERE, "pfpx_golden.npz"), **data)
    print("wrote", os.path.join(HERE, "pfpx_golden.npz"), sorted(data))


if __name__ == "__main__":
    main()
