"""The CUDA path on the reference's own fixtures, under the reference's gate.

The reference's acceptance test for a solver build is
`parity/compare_parity.py DIR_A DIR_B` exiting 0 on the outputs of
`--single-pass --eps 0 --no-theta` for BR1, BR2, BR3 and SYN1
(parity/compare_parity.py:16-41; outputs checked in under
parity/ref_{cpu,host,gpu}/). Here the plp_gpu CLI in each of its modes
writes those four JSON files into a directory and the gate (restated in
tests/parity_gate.py, checked against the reference script on the CPU)
must pass against the CPython, g++ and plain-CUDA outputs alike.

Beyond the gate, every instance of the reference's data/manifest.json (the
set tests/test_solver.py:288-302 smoke-tests) and SYN1 is decoded on the
GPU and compared with the reference g++ build (tests/golden/br.jsonl):
seed 0 at eps 0 in full, and seeds 0..15 at eps 0.3 / theta 0.9 through the
CLI's --device mode and through one batched library solve. The eps-0
packings also pass the reference's validity checks (inside the container,
no overlaps, final-state support >= 0.5).
"""
import json
import os
import subprocess

import pytest

import plpb200 as P
from conftest import GOLDEN
from parity_gate import compare_dirs, row_digest

FIX = os.path.join(GOLDEN, "reference")
PARITY = os.path.join(FIX, "parity")
NAMES = ["BR1", "BR2", "BR3", "SYN1"]
GATE_FLAGS = ["--single-pass", "--eps", "0", "--no-theta"]
pytestmark = pytest.mark.gpu


def br_rows(case):
    return [r for r in map(json.loads, open(os.path.join(GOLDEN, "br.jsonl"))) if r["case"] == case]


def inst_path(row):
    return os.path.join(FIX, "data", row["file"])


def cli(args):
    r = subprocess.run([P.CLI_PATH] + args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def cli_rows(path, flags, mode):
    """JSON objects of one CLI run: the single result, or the wrapper's rows."""
    out = json.loads(cli([path, "--json"] + flags + mode))
    return out["rows"] if "rows" in out else [out]


def check_valid(placements, L, W, H):
    """The reference's smoke checks (tests/test_solver.py:291-301)."""
    boxes = [p[1:] for p in placements]
    for x, y, z, w, d, h in boxes:
        assert 0 <= x and x + w <= L and 0 <= y and y + d <= W and 0 <= z and z + h <= H
    for i, a in enumerate(boxes):
        for b in boxes[i + 1:]:
            assert not (a[0] < b[0] + b[3] and b[0] < a[0] + a[3] and a[1] < b[1] + b[4]
                        and b[1] < a[1] + a[4] and a[2] < b[2] + b[5] and b[2] < a[2] + a[5])
    for x, y, z, w, d, h in boxes:
        if z == 0:
            continue
        s = sum(max(0, min(x + w, b[0] + b[3]) - max(x, b[0])) * max(0, min(y + d, b[1] + b[4]) - max(y, b[1]))
                for b in boxes if b[2] + b[5] == z)
        assert 2 * s >= w * d


@pytest.mark.parametrize("mode", [[], ["--plain"], ["--device", "4"], ["--batch", "4"]],
                         ids=["persistent", "plain", "device4", "batch4"])
def test_plp_gpu_passes_the_reference_parity_gate(tmp_path, mode):
    rows = {r["name"]: r for r in br_rows("eps0")}
    for n in NAMES:
        out = cli_rows(inst_path(rows[n]), GATE_FLAGS, mode)[0]     # row 0 = seed 0
        (tmp_path / f"{n}.json").write_text(json.dumps(out))
    for build in ("ref_cpu", "ref_host", "ref_gpu"):
        rc, text = compare_dirs(str(tmp_path), os.path.join(PARITY, build))
        assert rc == 0, f"{build}:\n{text}"
        assert text == "".join(f"{n} MATCH\n" for n in NAMES) + "RESULT: ALL MATCH\n"


def test_every_reference_instance_eps0_matches_reference_host_and_is_valid():
    rows = br_rows("eps0")
    assert len(rows) == 20
    for r in rows:
        got = cli_rows(inst_path(r), GATE_FLAGS, [])[0]
        got.pop("time_s")
        assert got == r["expected"][0], r["name"]
        (L, W, H), _, _ = P.Instance.load(inst_path(r)).info()
        check_valid(got["placements"], L, W, H)


def test_every_reference_instance_eps03_seeds_0_15_device_mode():
    for r in br_rows("eps03"):
        out = cli_rows(inst_path(r), ["--single-pass", "--seed", "0"], ["--device", "16"])
        assert len(out) == 16
        assert [row_digest(o) for o in out] == [e[0] for e in r["restarts"]], r["name"]
        first = dict(out[0])
        first.pop("time_s")
        assert first == r["first"]


def test_every_reference_instance_eps03_one_batched_solve():
    rows = br_rows("eps03")
    insts = [P.Instance.load(inst_path(r)) for r in rows]
    with P.Handle() as h:
        res = h.solve(insts, P.make_opts(seed=0, restarts=16))
    for r, got in zip(rows, res):
        digests = [row_digest(json.loads(got.json(k))) for k in range(16)]
        assert digests == [e[0] for e in r["restarts"]], r["name"]
