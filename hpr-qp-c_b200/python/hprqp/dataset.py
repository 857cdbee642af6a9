"""Solve every MPS file of a folder and write the result table.

``python -m hprqp.dataset DATA_DIR RESULT_DIR [options]`` writes
``RESULT_DIR/HPRQP_result.csv`` and appends to ``RESULT_DIR/HPRQP_log.txt``
in the layout of the reference's dataset runner (scripts/run_dataset.py):
one row per file with the columns of its ``FIELDNAMES`` (lines 24-43), then
an ``SGM10`` row of shifted geometric means (shift 10) and a ``solved`` row
of counts, computed by the same rules (``write_csv``, lines 164-215), so the
tables of both can be compared line by line.  A rerun keeps the rows of
files whose status is already final and solves the rest (lines 251-263).

The reference starts its solve_qp program once per file and parses what it
prints; here each file is read with ``build_from_mps`` and solved in this
process.  Per file by default (one ``solve_gpu`` call, the reference's
path), or, with ``--batch``, all files of the folder as one batch in one
persistent kernel (``hprqp_batch.h``; ``alg_time`` is then the instance's
own time on its CTA, ``hprqp_batch_get_times``, and the ``iter_4`` /
``iter_6`` columns stay empty because the batch does not record them).

Differences from the reference's table: a file the reader rejects gets the
reader's status name (``INVALID_ARGUMENT``, ...) where the reference writes
``EXIT_<code>``; ``gram_active``, ``polish_attempts`` and
``polish_accepted`` are 0 (no Gram path and no polishing here).  As in the
reference, ``input_format`` is ``mps_qcmatrix_v1`` (the reader lifts
diagonal QCMATRIX rows to second-order cones) and ``row_cones`` counts the
lifted cones.  With ``--batch``, files whose models have cones are solved
one by one (the batch kernel takes QPs only).
"""
from __future__ import annotations

import argparse
import csv
import math
import sys
import time
from datetime import datetime
from pathlib import Path
from typing import Dict, Iterable, List, Optional

CSV_NAME = "HPRQP_result.csv"
LOG_NAME = "HPRQP_log.txt"
SUMMARY_NAMES = ("SGM10", "solved")
SOLVED = ("OPTIMAL", "polished_optimal")
FINAL = SOLVED + ("OK", "MAX_ITER", "TIME_LIMIT")
INPUT_FORMAT = "mps_qcmatrix_v1"
FIELDNAMES = ["name", "iter", "alg_time", "res", "primal_obj", "gap", "status", "iter_4", "time_4", "iter_6",
              "time_6", "process_time", "total_time", "gram_active", "polish_attempts", "polish_accepted",
              "input_format", "row_cones"]


def _g(v: float) -> str:
    return f"{v:.12g}"


def shifted_geomean(values: Iterable[float], shift: float = 10.0) -> str:
    """exp(mean(log(v + shift))) - shift, as text; empty for no values."""
    vals = list(values)
    if not vals:
        return ""
    return _g(math.exp(sum(math.log(v + shift) for v in vals) / len(vals)) - shift)


def _num(row: Dict[str, str], key: str, as_int: bool = False) -> Optional[float]:
    text = row.get(key) or ""
    try:
        v = float(text)
    except ValueError:
        return None
    return float(int(v)) if as_int else v


def summary_rows(rows: List[Dict[str, str]], time_limit: float) -> List[Dict[str, str]]:
    """The SGM10 and solved rows below the per-file rows."""
    def column(key, as_int=False):
        return [v for v in (_num(r, key, as_int) for r in rows) if v is not None]

    sgm = {"name": "SGM10", "res": "", "primal_obj": "", "gap": "", "status": ""}
    solved = {"name": "solved", "iter": "", "res": "", "primal_obj": "", "gap": "", "status": "", "iter_4": "",
              "iter_6": ""}
    for key, as_int in (("iter", True), ("iter_4", True), ("time_4", False), ("iter_6", True), ("time_6", False)):
        sgm[key] = shifted_geomean(column(key, as_int))
    n_solved = sum(r.get("status") in SOLVED for r in rows)
    solved["time_4"] = str(sum(v < time_limit for v in column("time_4")))
    solved["time_6"] = str(sum(v < time_limit for v in column("time_6")))
    # clocks: an unsolved file counts as the time limit; a solved file
    # without a usable clock leaves the mean empty
    for clock in ("alg_time", "total_time", "process_time"):
        vals = [(_num(r, clock) if r.get("status") in SOLVED else time_limit) for r in rows]
        ok = all(v is not None and math.isfinite(v) and v >= 0 for v in vals)
        sgm[clock] = shifted_geomean(vals) if ok else ""
        solved[clock] = str(n_solved)
    return [sgm, solved]


def write_table(path: Path, rows: List[Dict[str, str]], time_limit: float) -> None:
    with path.open("w", newline="", encoding="ascii") as f:
        w = csv.DictWriter(f, fieldnames=FIELDNAMES, extrasaction="ignore")
        w.writeheader()
        w.writerows(rows)
        w.writerows(summary_rows(rows, time_limit))


def read_table(path: Path) -> List[Dict[str, str]]:
    if not path.exists():
        return []
    with path.open(newline="") as f:
        return [r for r in csv.DictReader(f) if r.get("name", "") not in SUMMARY_NAMES]


def has_qcmatrix(path: Path) -> bool:
    with path.open() as f:
        return any(line.split(maxsplit=1)[:1] == ["QCMATRIX"] for line in f)


def keep_previous(row: Dict[str, str], path: Path) -> bool:
    """A previous row stands if its status is final and it was made by a
    reader that reads QCMATRIX sections, or its file has none (the
    reference's can_resume, scripts/run_dataset.py:118-122)."""
    return row.get("status") in FINAL and (row.get("input_format") == INPUT_FORMAT or not has_qcmatrix(path))


def _row(name: str, **kw) -> Dict[str, str]:
    row = {k: "" for k in FIELDNAMES}
    row.update(name=name, gram_active="0", polish_attempts="0", polish_accepted="0", input_format=INPUT_FORMAT,
               row_cones="0")
    row.update({k: v if isinstance(v, str) else _g(v) if isinstance(v, float) else str(v) for k, v in kw.items()})
    return row


def _log(path: Path, text: str) -> None:
    with path.open("a", encoding="ascii", errors="replace") as f:
        f.write(text if text.endswith("\n") else text + "\n")


def _params(args):
    from . import Parameters

    p = Parameters(verbose=bool(args.verbose))
    for key in ("stoptol", "max_iter", "time_limit", "check_iter", "print_frequency", "device_number",
                "use_scaling", "spmv_mode_q", "spmv_mode_a"):
        v = getattr(args, key, None)
        if v is not None:
            getattr(p, "set_" + key)(v)
    return p


def _read(path: Path, log: Path):
    """(model, None) or (None, status name) for a file the reader rejects."""
    from . import read_from_mps, status_name

    try:
        return read_from_mps(path), None
    except RuntimeError as e:
        text = str(e)
        status = next((status_name(c) for c in range(9) if text.endswith(status_name(c))), "READ_FAILED")
        _log(log, f"read failed: {text}")
        return None, status


def solve_each(paths: List[Path], args, log: Path) -> List[Dict[str, str]]:
    """One solve_gpu call per file (the reference's path)."""
    rows = []
    for i, path in enumerate(paths, 1):
        _log(log, f"[{datetime.now():%Y-%m-%d %H:%M:%S}] solving problem {i}: {path.name}")
        t0 = time.perf_counter()
        model, failed = _read(path, log)
        if model is None:
            rows.append(_row(path.name, status=failed, process_time=time.perf_counter() - t0))
            continue
        rows.append(_solve_model(path.name, model, args, log, t0))
    return rows


def _solve_model(name: str, model, args, log: Path, t0: float) -> Dict[str, str]:
    from . import optimize

    t1 = time.perf_counter()
    r = optimize(model, _params(args))
    t2 = time.perf_counter()
    _log(log, f"iter: {r.iter}\ntime: {r.time:.12g}\nresidual: {r.residual:.12g}\nobjective: "
              f"{r.objective:.12g}\ngap: {r.gap:.12g}\nstatus: {r.status}")
    return _row(name, iter=r.iter, alg_time=r.time, res=r.residual, primal_obj=r.objective, gap=r.gap,
                status=r.status, iter_4=r.iter_4, time_4=r.time_4, iter_6=r.iter_6, time_6=r.time_6,
                process_time=t2 - t0, total_time=t2 - t1, row_cones=int(model._struct().num_row_cones))


def solve_batched(paths: List[Path], args, log: Path) -> List[Dict[str, str]]:
    """Every readable file as one instance of one batch (hprqp_batch.h)."""
    from . import status_name
    from .batch import Batch

    rows: Dict[str, Dict[str, str]] = {}
    insts, t_read = [], {}
    for path in paths:
        t0 = time.perf_counter()
        model, failed = _read(path, log)
        if model is None:
            rows[path.name] = _row(path.name, status=failed, process_time=time.perf_counter() - t0)
            continue
        st = model._struct()
        if st.num_row_cones or st.num_var_cones:
            _log(log, f"{path.name}: cone model, solved on its own")
            rows[path.name] = _solve_model(path.name, model, args, log, t0)
            continue
        insts.append(model.to_instance(path.name))
        t_read[path.name] = time.perf_counter() - t0
    if insts:
        kw = {k: getattr(args, k) for k in ("stoptol", "max_iter", "time_limit", "check_iter", "print_frequency",
                                             "use_scaling") if getattr(args, k, None) is not None}
        t1 = time.perf_counter()
        b = Batch(insts, device_number=args.device_number or 0)
        try:
            b.solve(**kw)
            res = b.results(vectors=False)
        finally:
            b.close()
        total = time.perf_counter() - t1
        _log(log, f"[{datetime.now():%Y-%m-%d %H:%M:%S}] batch of {len(insts)} files: launch "
                  f"{res.solve_ms / 1e3:.6g} s, create + solve + results {total:.6g} s")
        for k, inst in enumerate(insts):
            st = status_name(int(res.status[k]))
            _log(log, f"{inst.name}: iter {int(res.iter[k])} time {res.seconds[k]:.6g} residual "
                      f"{res.residual[k]:.6g} objective {res.objective[k]:.12g} status {st}")
            rows[inst.name] = _row(inst.name, iter=int(res.iter[k]), alg_time=float(res.seconds[k]),
                                   res=float(res.residual[k]), primal_obj=float(res.objective[k]),
                                   gap=float(res.gap[k]), status=st, process_time=t_read[inst.name] + total,
                                   total_time=total)
    return [rows[p.name] for p in paths]


def run(data_path, result_path, args) -> int:
    data, out = Path(data_path), Path(result_path)
    if not data.is_dir():
        print(f"dataset folder not found: {data}", file=sys.stderr)
        return 1
    out.mkdir(parents=True, exist_ok=True)
    table, log = out / CSV_NAME, out / LOG_NAME
    rows = read_table(table)
    index = {r["name"]: i for i, r in enumerate(rows) if r.get("name")}
    files = sorted(p for p in data.iterdir() if p.is_file() and p.suffix.lower() == ".mps")
    todo = [p for p in files if not (p.name in index and keep_previous(rows[index[p.name]], p))]
    new = (solve_batched if args.batch else solve_each)(todo, args, log) if todo else []
    for row in new:
        if row["name"] in index:
            rows[index[row["name"]]] = row
        else:
            index[row["name"]] = len(rows)
            rows.append(row)
    write_table(table, rows, args.time_limit)
    return 0


def parse_args(argv=None) -> argparse.Namespace:
    ap = argparse.ArgumentParser(description="Solve every .mps file of a folder; write HPRQP_result.csv.")
    ap.add_argument("data_path", help="folder of .mps files")
    ap.add_argument("result_path", help="folder for HPRQP_result.csv and HPRQP_log.txt")
    ap.add_argument("--batch", action="store_true", help="solve all files as one batch (one kernel launch)")
    ap.add_argument("--max-iter", type=int)
    ap.add_argument("--stoptol", type=float)
    ap.add_argument("--check-iter", type=int)
    ap.add_argument("--print-frequency", type=int)
    ap.add_argument("--time-limit", type=float, default=3600.0)
    ap.add_argument("--verbose", type=int, default=0)
    ap.add_argument("--use-gpu", type=int, choices=[1], help="accepted for the reference's flags; GPU only")
    ap.add_argument("--device-number", type=int)
    ap.add_argument("--spmv-mode-q", choices=["auto", "cusparse", "customized"])
    ap.add_argument("--spmv-mode-a", choices=["auto", "cusparse", "customized"])
    ap.add_argument("--use-scaling", type=int)
    return ap.parse_args(argv)


def main(argv=None) -> int:
    args = parse_args(argv)
    return run(args.data_path, args.result_path, args)


if __name__ == "__main__":
    raise SystemExit(main())
