"""Record the C symbols the reference's own language bindings bind: every
``hprqp_*`` name in its Python package (python/src/hprqp/__init__.py) and
its Julia package (julia/src/*.jl).  Writes reference_ffi_symbols.json
beside this file; tests/test_abi.py requires this library to export each
one, so both wrappers can load it unchanged.

    python tests/golden/make_ffi_symbols.py <reference checkout>
"""
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
NAME = re.compile(r"\bhprqp_[a-z0-9_]+\b")


def names(paths):
    out = set()
    for p in paths:
        out |= set(NAME.findall(p.read_text()))
    return sorted(out)


if __name__ == "__main__":
    ref = Path(sys.argv[1])
    data = {"python": names([ref / "python" / "src" / "hprqp" / "__init__.py"]),
            "julia": names(sorted((ref / "julia" / "src").glob("*.jl")))}
    (HERE / "reference_ffi_symbols.json").write_text(json.dumps(data, indent=1) + "\n")
    print({k: len(v) for k, v in data.items()})
