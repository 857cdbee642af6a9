"""The MPS reader on mutated files (lines dropped, repeated, truncated,
tokens replaced by section names, bound types, extreme or malformed
numbers): every file is either read or rejected with a status, never a
crash.  Seeded; the same mutations were also run against the library built
with AddressSanitizer + UndefinedBehaviorSanitizer
(``python hpr-qp-c_b200/build.py --sanitize``) without a report."""
from __future__ import annotations

import random

from mps_cases import malformed, malformed_qcqp, random_mps, random_qcqp_mps

TOKENS = ["ROWS", "COLUMNS", "RHS", "RANGES", "BOUNDS", "QUADOBJ", "QMATRIX", "QCMATRIX", "ENDATA", "NAME",
          "OBJSENSE", "MAX", "MIN", " N", " E", " L", " G", "UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI",
          "'MARKER'", "'INTORG'", "'INTEND'", "1e308", "-1e308", "nan", "inf", "1D5", "0", "-0", "x" * 300, "\t"]


def _mutate(rng, text):
    lines = text.splitlines()
    for _ in range(rng.randint(1, 6)):
        op = rng.randrange(6)
        i = rng.randrange(len(lines)) if lines else 0
        if op == 0 and lines:
            del lines[i]
        elif op == 1 and lines:
            lines.insert(i, lines[rng.randrange(len(lines))])
        elif op == 2 and lines and lines[i].split():
            t = lines[i].split()
            t[rng.randrange(len(t))] = rng.choice(TOKENS)
            lines[i] = ("    " if lines[i].startswith(" ") else "") + " ".join(t)
        elif op == 3:
            lines.insert(i, rng.choice(TOKENS) + " " + rng.choice(TOKENS))
        elif op == 4 and lines:
            lines[i] = lines[i][:rng.randrange(len(lines[i]) + 1)]
        else:
            lines.insert(i, "    " + " ".join(rng.choice(TOKENS) for _ in range(rng.randint(1, 7))))
    return "\n".join(lines) + ("\n" if rng.random() < 0.9 else "")


def test_mutated_files_are_read_or_rejected(engine_lib, tmp_path):
    hprqp = engine_lib
    rng = random.Random(20261204)
    seeds = [random_mps(s, n=6 + s % 5, m=4 + s % 4, quad=q) for s in range(4) for q in ("QUADOBJ", "QMATRIX", "")]
    seeds += [random_qcqp_mps(s) for s in range(3)] + list(malformed().values()) + list(malformed_qcqp().values())
    read = rejected = 0
    p = tmp_path / "f.mps"
    for _ in range(400):
        p.write_text(_mutate(rng, rng.choice(seeds)))
        try:
            model = hprqp.read_from_mps(p)
            assert model.num_variables >= 0
            read += 1
        except RuntimeError as err:
            assert "failed with status" in str(err)
            rejected += 1
    assert read > 0 and rejected > 0
