"""The dataset runner's table and resume rules (hprqp.dataset), on CPU.

The table must be the reference runner's, text for text: the golden files
were written by the reference's own write_csv (scripts/run_dataset.py) from
the rows in dataset_rows.json (tests/golden/make_dataset_table.py)."""
from __future__ import annotations

import json
from pathlib import Path

import pytest

from hprqp import dataset

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("limit,name", [(3600.0, "dataset_table.csv"), (10.0, "dataset_table_limit10.csv")])
def test_table_matches_reference_writer(tmp_path, limit, name):
    rows = json.loads((GOLDEN / "dataset_rows.json").read_text())
    out = tmp_path / "t.csv"
    dataset.write_table(out, rows, limit)
    assert out.read_text() == (GOLDEN / name).read_text()


def test_shifted_geomean():
    assert dataset.shifted_geomean([]) == ""
    assert dataset.shifted_geomean([5.0]) == "5"
    assert float(dataset.shifted_geomean([0.0, 30.0])) == pytest.approx((10.0 * 40.0) ** 0.5 - 10.0)


def test_read_table_drops_summary_rows(tmp_path):
    rows = json.loads((GOLDEN / "dataset_rows.json").read_text())
    out = tmp_path / "t.csv"
    dataset.write_table(out, rows, 3600.0)
    back = dataset.read_table(out)
    assert [r["name"] for r in back] == [r["name"] for r in rows]
    assert back[2]["status"] == "TIME_LIMIT"


def _args(**kw):
    return dataset.parse_args(["in", "out"] + [f"--{k.replace('_', '-')}={v}" for k, v in kw.items()])


def test_resume_solves_only_what_is_not_final(tmp_path, monkeypatch):
    data = tmp_path / "data"
    data.mkdir()
    (data / "a.mps").write_text("NAME A\nENDATA\n")
    (data / "b.mps").write_text("NAME B\nENDATA\n")
    (data / "q.mps").write_text("NAME Q\nQCMATRIX c1\nENDATA\n")
    (data / "notes.txt").write_text("not an MPS file\n")
    calls = []
    status = {"a.mps": "OPTIMAL", "b.mps": "NOT_IMPLEMENTED", "q.mps": "OPTIMAL"}

    def fake(paths, args, log):
        calls.append([p.name for p in paths])
        return [dataset._row(p.name, iter=10, alg_time=0.5, status=status[p.name], process_time=0.6,
                             total_time=0.55) for p in paths]

    monkeypatch.setattr(dataset, "solve_each", fake)
    out = tmp_path / "out"
    assert dataset.run(data, out, _args()) == 0
    assert calls == [["a.mps", "b.mps", "q.mps"]]
    # a.mps and q.mps are final; b.mps failed
    status["b.mps"] = "OPTIMAL"
    assert dataset.run(data, out, _args()) == 0
    assert calls[1] == ["b.mps"]
    # a QCMATRIX file's row from a reader that did not read QCMATRIX (no
    # input_format) does not stand, as in the reference
    rows = dataset.read_table(out / dataset.CSV_NAME)
    for r in rows:
        if r["name"] == "q.mps":
            r["input_format"] = ""
    dataset.write_table(out / dataset.CSV_NAME, rows, 3600.0)
    assert dataset.run(data, out, _args()) == 0
    assert calls[2] == ["q.mps"]
    rows = dataset.read_table(out / dataset.CSV_NAME)
    assert [r["name"] for r in rows] == ["a.mps", "b.mps", "q.mps"]
    assert all(r["status"] == "OPTIMAL" for r in rows)
    text = (out / dataset.CSV_NAME).read_text().splitlines()
    assert text[0].split(",") == dataset.FIELDNAMES
    assert text[-1].startswith("solved,,3,")


def test_batch_flag_selects_the_batched_solver(tmp_path, monkeypatch):
    data = tmp_path / "data"
    data.mkdir()
    (data / "a.mps").write_text("NAME A\nENDATA\n")
    seen = []
    monkeypatch.setattr(dataset, "solve_batched",
                        lambda paths, args, log: seen.append("batch") or [dataset._row("a.mps", status="OPTIMAL")])
    monkeypatch.setattr(dataset, "solve_each",
                        lambda paths, args, log: seen.append("each") or [dataset._row("a.mps", status="OPTIMAL")])
    dataset.run(data, tmp_path / "o1", dataset.parse_args(["x", "y", "--batch"]))
    dataset.run(data, tmp_path / "o2", dataset.parse_args(["x", "y"]))
    assert seen == ["batch", "each"]


def test_missing_folder(tmp_path):
    assert dataset.run(tmp_path / "nope", tmp_path / "out", _args()) == 1


def test_failed_status_and_missing_clocks(tmp_path):
    """the reference's tests/test_dataset.py:110-120: an unsolved file counts
    as the time limit, a solved file without a process clock empties that
    mean, and the solved count is 1"""
    out = tmp_path / "a.csv"
    dataset.write_table(out, [{"name": "success", "status": "OPTIMAL", "alg_time": "1200"},
                              {"name": "fail", "status": "TIME_LIMIT", "alg_time": "2"}], 1000)
    import csv

    with out.open() as f:
        rows = list(csv.DictReader(f))
    assert float(rows[-2]["alg_time"]) == pytest.approx((1210 * 1010) ** 0.5 - 10, abs=1e-7)
    assert rows[-2]["process_time"] == ""
    assert rows[-1]["alg_time"] == "1"


def test_legacy_qcqp_rows_do_not_stand(tmp_path):
    """the reference's tests/test_dataset.py:17-26"""
    path = tmp_path / "qc.mps"
    path.write_text("NAME TEST\nQCMATRIX QC\n X X 0.5\nENDATA\n")
    old = {"status": "OPTIMAL"}
    assert not dataset.keep_previous(old, path)
    old["input_format"] = dataset.INPUT_FORMAT
    assert dataset.keep_previous(old, path)
    old["status"] = "EXIT_1"
    assert not dataset.keep_previous(old, path)
