"""Writes tests/golden/project_report_keys.json: the keys of the report dict
that the reference's CartesianFluidSolver.project returns with read_report
(simulation_core/fluid.py, the dict literal at the end of project), read
from the reference's source as text.

    python tests/golden/make_report_keys.py <reference tree>
"""

from __future__ import annotations

import ast
import json
import sys
from pathlib import Path


def report_keys(fluid_py: Path) -> list[str]:
    tree = ast.parse(fluid_py.read_text())
    for node in ast.walk(tree):
        if isinstance(node, ast.ClassDef) and node.name == "CartesianFluidSolver":
            for fn in node.body:
                if isinstance(fn, ast.FunctionDef) and fn.name == "project":
                    returns = [r for r in ast.walk(fn) if isinstance(r, ast.Return) and isinstance(r.value, ast.Dict)]
                    largest = max(returns, key=lambda r: len(r.value.keys))
                    return [k.value for k in largest.value.keys if isinstance(k, ast.Constant)]
    raise SystemExit("CartesianFluidSolver.project not found")


def main(argv: list[str]) -> None:
    if len(argv) != 2:
        raise SystemExit(__doc__)
    keys = report_keys(Path(argv[1]) / "simulation_core" / "fluid.py")
    out = Path(__file__).with_name("project_report_keys.json")
    out.write_text(json.dumps({"source": "simulation_core/fluid.py CartesianFluidSolver.project", "keys": keys},
                              indent=1) + "\n")
    print(f"{len(keys)} keys -> {out}")


if __name__ == "__main__":
    main(sys.argv)
