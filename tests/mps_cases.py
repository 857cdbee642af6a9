"""Seeded MPS text generator for the MPS-reader tests (this project's own
files: random QPs written in free MPS with every construct the reader
accepts -- N/E/L/G rows, RANGES of both signs on every row kind, an
objective constant in RHS, all continuous bound types, one or two pairs per
line, Fortran 'D' exponents, comments, a second RHS/BOUNDS set and a second
N row that the reader must ignore -- plus malformed variants)."""
from __future__ import annotations

import numpy as np


def _num(rng, v):
    r = rng.random()
    if r < 0.15:
        return f"{v:.17g}".replace("e", "D") if "e" in f"{v:.17g}" else f"{v:.17g}D0"
    if r < 0.3:
        return f"{v:.6e}"
    return repr(float(v))


def random_mps(seed: int, n: int = 12, m: int = 8, quad: str = "QUADOBJ") -> str:
    rng = np.random.default_rng(seed)
    rows = [f"R{i}" for i in range(m)]
    kinds = [rng.choice(["E", "L", "G"]) for _ in range(m)]
    cols = [f"X{j}" for j in range(n)]
    A = (rng.random((m, n)) < 0.35) * np.round(rng.standard_normal((m, n)), 3)
    c = np.round(rng.standard_normal(n), 4)
    out = ["* generated", "NAME          GEN%d" % seed, "ROWS", " N  COST"]
    out += [f" {k}  {r}" for k, r in zip(kinds, rows)]
    out += [" N  EXTRA"]  # a second objective row: ignored
    out.append("COLUMNS")
    for j, col in enumerate(cols):
        pairs = [("COST", c[j])] if c[j] != 0 else []
        pairs += [(rows[i], A[i, j]) for i in range(m) if A[i, j] != 0]
        if rng.random() < 0.3:
            pairs.append(("EXTRA", 1.0))
        if not pairs:
            pairs = [("COST", 0.0)]
        k = 0
        while k < len(pairs):
            if k + 1 < len(pairs) and rng.random() < 0.5:
                out.append(f"    {col}  {pairs[k][0]}  {_num(rng, pairs[k][1])}  {pairs[k + 1][0]}  "
                           f"{_num(rng, pairs[k + 1][1])}")
                k += 2
            else:
                out.append(f"    {col}\t{pairs[k][0]}\t{_num(rng, pairs[k][1])}")
                k += 1
    out.append("RHS")
    out.append(f"    RHS1  COST  {_num(rng, round(rng.standard_normal(), 3))}")
    for i, r in enumerate(rows):
        if rng.random() < 0.8:
            out.append(f"    RHS1  {r}  {_num(rng, round(rng.standard_normal() * 2, 3))}")
    out.append(f"    RHS2  {rows[0]}  99")  # second set: skipped
    out.append("RANGES")
    for i, r in enumerate(rows):
        if rng.random() < 0.5:
            out.append(f"    RNG  {r}  {_num(rng, round(rng.standard_normal() * 3, 3))}")
    out.append("BOUNDS")
    for j, col in enumerate(cols):
        t = rng.integers(0, 9)
        v = round(float(rng.standard_normal() * 4), 3)
        if t == 0:
            out.append(f" UP BND  {col}  {_num(rng, v)}")  # negative -> lower becomes -inf
        elif t == 1:
            out.append(f" LO BND  {col}  {_num(rng, v)}")
        elif t == 2:
            out.append(f" FX BND  {col}  {_num(rng, v)}")
        elif t == 3:
            out.append(f" FR BND  {col}")
        elif t == 4:
            out.append(f" MI BND  {col}")
        elif t == 5:
            out.append(f" PL BND  {col}")
        elif t == 6:
            out.append(f" LO BND  {col}  {_num(rng, -abs(v))}")
            out.append(f" UP BND  {col}  {_num(rng, abs(v) + 1)}")
        # t >= 7: default bounds
    out.append(f" UP OTHER  {cols[0]}  5")  # second set: skipped
    if quad:
        out.append(quad)
        M = np.round(rng.standard_normal((n, n // 2)), 2)
        Q = M @ M.T + np.eye(n) * 0.5
        Q = np.round(Q, 3)
        Q = 0.5 * (Q + Q.T)
        mask = rng.random((n, n)) < 0.3
        mask = mask | mask.T | np.eye(n, dtype=bool)
        for i in range(n):
            for j in range(n):
                if not mask[i, j] or Q[i, j] == 0:
                    continue
                if quad == "QUADOBJ" and j > i:
                    continue
                out.append(f"    {cols[i]}  {cols[j]}  {_num(rng, Q[i, j])}")
    out.append("ENDATA")
    return "\n".join(out) + "\n"


def malformed() -> dict:
    """name -> MPS text that both readers must reject."""
    base = ["NAME T", "ROWS", " N obj", " L c1", "COLUMNS", "    x obj 1 c1 2", "RHS", "    rhs c1 3"]
    return {
        "unknown_row": "\n".join(base[:5] + ["    x nope 1"] + base[6:] + ["ENDATA"]) + "\n",
        "bad_number": "\n".join(base[:5] + ["    x obj 1.2.3"] + base[6:] + ["ENDATA"]) + "\n",
        "no_endata": "\n".join(base) + "\n",
        "maximize": "\n".join(["NAME T", "OBJSENSE", "    MAX"] + base[1:] + ["ENDATA"]) + "\n",
        "integer": "\n".join(base[:5] + ["    M1 'MARKER' 'INTORG'", "    x obj 1 c1 2",
                                         "    M2 'MARKER' 'INTEND'"] + base[6:] + ["ENDATA"]) + "\n",
        "dup_row": "\n".join(base[:4] + [" L c1"] + base[4:] + ["ENDATA"]) + "\n",
        "unknown_bound_col": "\n".join(base + ["BOUNDS", " UP b y 3", "ENDATA"]) + "\n",
        "binary": "\n".join(base + ["BOUNDS", " BV b x", "ENDATA"]) + "\n",
        "asym_qmatrix": "\n".join(base[:5] + ["    x obj 1 c1 2", "    y c1 1"] + base[6:] +
                                   ["QMATRIX", "    x y 1", "    y x 2", "ENDATA"]) + "\n",
    }


def write_instance(inst) -> str:
    """A QPInstance as free MPS (QUADOBJ lower triangle; ranged rows as G
    rows with a RANGES entry, so their upper side is AL + (AU - AL))."""
    import numpy as np

    n, m = inst.n, inst.m
    out = ["NAME INST", "ROWS", " N OBJ"]
    kinds = []
    for i in range(m):
        lo, up = inst.AL[i], inst.AU[i]
        k = "E" if lo == up else ("L" if np.isneginf(lo) else "G")
        kinds.append(k)
        out.append(f" {k} R{i}")
    out.append("COLUMNS")
    at = inst.A.to_scipy().T.tocsr()
    for j in range(n):
        out.append(f"    X{j} OBJ {float(inst.c[j])!r}")
        for e in range(at.indptr[j], at.indptr[j + 1]):
            out.append(f"    X{j} R{at.indices[e]} {float(at.data[e])!r}")
    out.append("RHS")
    if inst.obj_constant:
        out.append(f"    RHS OBJ {-float(inst.obj_constant)!r}")
    for i, k in enumerate(kinds):
        v = inst.AU[i] if k == "L" else inst.AL[i]
        if np.isfinite(v) and v != 0:
            out.append(f"    RHS R{i} {float(v)!r}")
    rng = [(i, float(inst.AU[i] - inst.AL[i])) for i, k in enumerate(kinds)
           if k == "G" and np.isfinite(inst.AU[i])]
    if rng:
        out.append("RANGES")
        out += [f"    RNG R{i} {v!r}" for i, v in rng]
    out.append("BOUNDS")
    for j in range(n):
        lo, up = float(inst.l[j]), float(inst.u[j])
        if np.isneginf(lo) and np.isposinf(up):
            out.append(f" FR BND X{j}")
            continue
        if np.isneginf(lo):
            out.append(f" MI BND X{j}")
        elif lo != 0.0:
            out.append(f" LO BND X{j} {lo!r}")
        if np.isfinite(up):
            out.append(f" UP BND X{j} {up!r}")
    out.append("QUADOBJ")
    q = inst.Q.to_scipy().tocsr()
    for i in range(n):
        for e in range(q.indptr[i], q.indptr[i + 1]):
            j = q.indices[e]
            if j <= i:
                out.append(f"    X{i} X{j} {float(q.data[e])!r}")
    out.append("ENDATA")
    return "\n".join(out) + "\n"


def random_qcqp_mps(seed: int, n: int = 8, m: int = 6) -> str:
    """A convex QCQP in free MPS: QUADOBJ diagonal objective, L and G rows
    with diagonal QCMATRIX blocks (positive on L rows, negative on G rows,
    a repeated entry to be summed, a zero entry to be dropped), one block of
    zeros only (the row stays linear), an E row and a ranged row without
    quadratic terms; x = 0 is feasible."""
    rng = np.random.default_rng(seed)
    cols = [f"X{j}" for j in range(n)]
    kinds = ["L", "G", "L", "G", "E", "L"] + [rng.choice(["L", "G"]) for _ in range(m - 6)]
    A = (rng.random((m, n)) < 0.5) * np.round(rng.standard_normal((m, n)), 3)
    out = ["NAME QCQP%d" % seed, "ROWS", " N  OBJ"] + [f" {k}  R{i}" for i, k in enumerate(kinds)]
    out.append("COLUMNS")
    c = np.round(rng.standard_normal(n), 3)
    for j, col in enumerate(cols):
        out.append(f"    {col}  OBJ  {float(c[j])!r}")
        for i in range(m):
            if A[i, j] != 0:
                out.append(f"    {col}  R{i}  {float(A[i, j])!r}")
    out.append("RHS")
    for i, k in enumerate(kinds):
        v = {"L": 1.0 + rng.random(), "G": -1.0 - rng.random(), "E": 0.0}[k]
        out.append(f"    RHS  R{i}  {float(v)!r}")
    out += ["RANGES", "    RNG  R5  2.5"]
    out += ["BOUNDS"] + [f" LO BND {col} -2" for col in cols[: n // 2]] + [f" FR BND {col}" for col in cols[n // 2:]]
    out.append("QUADOBJ")
    out += [f"    {col}  {col}  {float(1.0 + rng.random())!r}" for col in cols]
    for i in range(4):
        sgn = 1.0 if kinds[i] == "L" else -1.0
        out.append(f"QCMATRIX  R{i}")
        for j in sorted(rng.choice(n, size=3, replace=False)):
            out.append(f"    X{j}  X{j}  {float(sgn * (0.5 + rng.random()))!r}")
        out.append(f"    X{j}  X{j}  {sgn * 0.25!r}")  # a second entry for the same column
        out.append(f"    X0  X1  0.0")  # an explicit zero off the diagonal: ignored
    out += [f"QCMATRIX  R{m - 1}", "    X2  X2  0.0"]  # zeros only: the row stays linear
    out.append("ENDATA")
    return "\n".join(out) + "\n"


def malformed_qcqp() -> dict:
    """name -> QCMATRIX misuse that both readers must reject."""
    head = ["NAME T", "ROWS", " N obj", " L c1", " G c2", " E c3", "COLUMNS", "    x obj 1 c1 1",
            "    x c2 1 c3 1", "    y c1 1 c2 1", "RHS", "    rhs c1 4 c2 -1", "    rhs c3 0.5"]
    end = ["ENDATA"]
    blocks = {
        "on_equality_row": ["QCMATRIX c3", "    x x 1"],
        "ranged_row": ["RANGES", "    rng c1 2", "QCMATRIX c1", "    x x 1"],
        "nonconvex_le": ["QCMATRIX c1", "    x x -1"],
        "nonconvex_ge": ["QCMATRIX c2", "    x x 1"],
        "off_diagonal": ["QCMATRIX c1", "    x y 1", "    y x 1"],
        "unknown_column": ["QCMATRIX c1", "    z z 1"],
        "objective_row": ["QCMATRIX obj", "    x x 1"],
        "duplicate_block": ["QCMATRIX c1", "    x x 1", "QCMATRIX c1", "    y y 1"],
        "bad_number": ["QCMATRIX c1", "    x x 1.2.3"],
        "two_fields": ["QCMATRIX c1", "    x 1"],
    }
    out = {k: "\n".join(head + v + end) + "\n" for k, v in blocks.items()}
    out["before_columns"] = "\n".join(["NAME T", "ROWS", " N obj", " L c1", "QCMATRIX c1", "    x x 1",
                                       "COLUMNS", "    x obj 1 c1 1", "ENDATA"]) + "\n"
    return out
