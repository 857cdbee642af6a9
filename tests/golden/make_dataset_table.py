"""Golden fixture for the dataset table: the reference's own write_csv
(scripts/run_dataset.py, imported from a checkout of the reference given as
the first argument) applied to fixed rows.  Writes dataset_rows.json (the
rows) and dataset_table.csv (the reference's table text) beside this file.

    python tests/golden/make_dataset_table.py <path of the reference checkout>
"""
import importlib.util
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
FIELDS = ["name", "iter", "alg_time", "res", "primal_obj", "gap", "status", "iter_4", "time_4", "iter_6",
          "time_6", "process_time", "total_time", "gram_active", "polish_attempts", "polish_accepted",
          "input_format", "row_cones"]


def row(name, it, t, status, it4, t4, it6, t6, pt, tt):
    r = dict.fromkeys(FIELDS, "")
    r.update(name=name, iter=it, alg_time=t, res="3.1e-07", primal_obj="-12.5", gap="1e-08", status=status,
             iter_4=it4, time_4=t4, iter_6=it6, time_6=t6, process_time=pt, total_time=tt, gram_active="0",
             polish_attempts="0", polish_accepted="0", input_format="mps", row_cones="0")
    return r


ROWS = [
    row("a.mps", "310", "0.0421", "OPTIMAL", "120", "0.02", "300", "0.04", "0.9", "0.05"),
    row("b.mps", "12000", "3.75", "OPTIMAL", "800", "0.3", "11000", "3.5", "4.1", "3.8"),
    row("c.mps", "100000", "3600.2", "TIME_LIMIT", "5000", "12.5", "", "", "3601", "3600.5"),
    row("d.mps", "", "", "NOT_IMPLEMENTED", "", "", "", "", "0.01", ""),
    row("e.mps", "50000", "88.1", "MAX_ITER", "2000", "5.5", "40000", "80.2", "90", "88.5"),
    row("f.mps", "7", "0.001", "OPTIMAL", "3", "0.0005", "7", "0.001", "", "0.002"),
]

if __name__ == "__main__":
    ref = Path(sys.argv[1]) / "scripts" / "run_dataset.py"
    spec = importlib.util.spec_from_file_location("ref_run_dataset", ref)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    (HERE / "dataset_rows.json").write_text(json.dumps(ROWS, indent=1) + "\n")
    for limit, name in ((3600.0, "dataset_table.csv"), (10.0, "dataset_table_limit10.csv")):
        mod.write_csv(HERE / name, [dict(r) for r in ROWS], limit)
    print("wrote", HERE / "dataset_rows.json", HERE / "dataset_table.csv", HERE / "dataset_table_limit10.csv")
