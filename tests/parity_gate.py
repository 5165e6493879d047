"""The reference's parity gate, restated for the tests (test infrastructure).

The reference accepts a solver build when `parity/compare_parity.py DIR_A
DIR_B [NAME ...]` exits 0 (parity/compare_parity.py:16-41): for every name
(default: every *.json stem in DIR_A) both JSON files are loaded, `time_s`
is removed from each (a file without it is an error), and the remaining
objects must be equal, floats included. It prints one `NAME MATCH` or
`NAME MISMATCH` line per name (a mismatch lists each differing field with
both values cut to 200 characters) and a final `RESULT:` line.

`compare_dirs` returns the same exit code and the same text, so a GPU test
can apply the reference's own acceptance rule on a machine where the
reference tree is absent; tests/test_parity_gate.py checks the two against
each other on the reference's fixtures wherever the reference is mounted.
"""
from __future__ import annotations

import hashlib
import json
import os


def row_digest(row: dict) -> str:
    """sha256 of one result row's JSON with time_s removed, keys sorted,
    compact separators: the form the digest fixtures in tests/golden/ use."""
    d = {k: v for k, v in row.items() if k != "time_s"}
    return hashlib.sha256(json.dumps(d, sort_keys=True, separators=(",", ":")).encode()).hexdigest()


def _load_without_time(path: str) -> dict:
    obj = json.load(open(path))
    del obj["time_s"]           # the reference pops it without a default
    return obj


def compare_dirs(dir_a: str, dir_b: str, names=None) -> tuple[int, str]:
    """(exit code, printed text) of the reference gate on DIR_A vs DIR_B."""
    if not names:
        names = sorted(f[:-len(".json")] for f in os.listdir(dir_a) if f.endswith(".json"))
    lines, all_match = [], True
    for name in names:
        a = _load_without_time(os.path.join(dir_a, name + ".json"))
        b = _load_without_time(os.path.join(dir_b, name + ".json"))
        if a == b:
            lines.append(f"{name} MATCH")
            continue
        all_match = False
        lines.append(f"{name} MISMATCH")
        for key in sorted(set(a) | set(b)):
            va, vb = a.get(key), b.get(key)
            if va != vb:
                lines += [f"  field: {key}", "    A: " + str(va)[:200], "    B: " + str(vb)[:200]]
    lines.append("RESULT: " + ("ALL MATCH" if all_match else "HAS MISMATCH"))
    return (0 if all_match else 1), "\n".join(lines) + "\n"
