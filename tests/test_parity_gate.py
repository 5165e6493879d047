"""The reference's parity gate and its own fixtures, on the CPU.

* The gate restatement (tests/parity_gate.py) gives the same exit code and
  the same text as the reference's parity/compare_parity.py on the
  reference's checked-in outputs and on altered copies of them (where the
  reference tree is mounted).
* The fixture copies under tests/golden/reference/ are byte-identical to
  the reference's data/ and parity/ files (where mounted).
* The reference's three checked-in builds (CPython, g++, plain CUDA) pass
  the gate against each other.
* The CPU oracle reproduces the reference g++ build on every instance of
  data/manifest.json (tests/test_solver.py:288-302 runs the same set) and on
  SYN1: seed 0 at --eps 0 --no-theta in full, and seeds 0..15 at eps 0.3 /
  theta 0.9 by row digest; its eps-0 outputs pass the gate against
  parity/ref_cpu and parity/ref_host.
"""
import json
import os
import shutil
import subprocess
import sys

import pytest

import oracle_py as O
from conftest import GOLDEN, REFERENCE, has_reference
from parity_gate import compare_dirs, row_digest

FIX = os.path.join(GOLDEN, "reference")
PARITY = os.path.join(FIX, "parity")
NAMES = ["BR1", "BR2", "BR3", "SYN1"]
REF_GATE = os.path.join(REFERENCE, "parity", "compare_parity.py")


def br_rows():
    return [json.loads(l) for l in open(os.path.join(GOLDEN, "br.jsonl"))]


def instance_text(file):
    return open(os.path.join(FIX, "data", file)).read()


def _mutated(tmp_path, src_dir, name, mutate):
    out = tmp_path / f"mut_{name}_{len(list(tmp_path.iterdir()))}"
    shutil.copytree(src_dir, out)
    p = out / f"{name}.json"
    d = json.load(open(p))
    mutate(d)
    p.write_text(json.dumps(d))
    return str(out)


@pytest.mark.skipif(not has_reference(), reason="reference tree not mounted")
def test_fixture_copies_are_byte_identical_to_the_reference():
    man = json.load(open(os.path.join(FIX, "data", "manifest.json")))["instances"]
    files = [e["file"] for e in man] + ["synthetic/SYN1.txt"]
    assert len(man) == 19
    for f in files:
        assert open(os.path.join(FIX, "data", f), "rb").read() == \
            open(os.path.join(REFERENCE, "data", f), "rb").read(), f
    for build in ("ref_cpu", "ref_host", "ref_gpu"):
        for n in NAMES:
            assert open(os.path.join(PARITY, build, n + ".json"), "rb").read() == \
                open(os.path.join(REFERENCE, "parity", build, n + ".json"), "rb").read()


@pytest.mark.skipif(not has_reference(), reason="reference tree not mounted")
def test_gate_restatement_matches_the_reference_script(tmp_path):
    cpu, host, gpu = (os.path.join(PARITY, b) for b in ("ref_cpu", "ref_host", "ref_gpu"))

    def bump_score(d):
        d["stability_score"] = d["stability_score"] + 1e-16 if d["stability_score"] else 1e-300

    def drop_box(d):
        d["placements"] = d["placements"][:-1]
        d["n_boxes"] -= 1

    def extra_key(d):
        d["extra"] = "x" * 300

    cases = [(cpu, host, []), (cpu, gpu, []), (host, gpu, ["BR2", "SYN1"]),
             (cpu, _mutated(tmp_path, host, "BR2", bump_score), []),
             (_mutated(tmp_path, cpu, "BR1", drop_box), host, ["BR1", "BR3"]),
             (cpu, _mutated(tmp_path, gpu, "SYN1", extra_key), [])]
    seen_rc = set()
    for a, b, names in cases:
        ref = subprocess.run([sys.executable, REF_GATE, a, b] + names, capture_output=True, text=True)
        rc, text = compare_dirs(a, b, names)
        assert (rc, text) == (ref.returncode, ref.stdout)
        seen_rc.add(rc)
    assert seen_rc == {0, 1}


def test_reference_builds_pass_the_gate_against_each_other():
    for a, b in (("ref_cpu", "ref_host"), ("ref_cpu", "ref_gpu")):
        rc, text = compare_dirs(os.path.join(PARITY, a), os.path.join(PARITY, b))
        assert rc == 0, text
        assert text.splitlines()[-1] == "RESULT: ALL MATCH"


def test_gate_reports_a_changed_float_and_a_missing_time(tmp_path):
    tmp = str(tmp_path / "host")
    shutil.copytree(os.path.join(PARITY, "ref_host"), tmp)
    p = os.path.join(tmp, "BR3.json")
    d = json.load(open(p))
    d["stability_score"] += 2 ** -52
    json.dump(d, open(p, "w"))
    rc, text = compare_dirs(os.path.join(PARITY, "ref_cpu"), tmp)
    assert rc == 1 and "BR3 MISMATCH\n  field: stability_score" in text
    d.pop("time_s")
    json.dump(d, open(p, "w"))
    with pytest.raises(KeyError):
        compare_dirs(os.path.join(PARITY, "ref_cpu"), tmp)


def test_oracle_eps0_on_every_reference_instance(tmp_path):
    rows = [r for r in br_rows() if r["case"] == "eps0"]
    assert len(rows) == 20
    for r in rows:
        inst = O.OInstance(instance_text(r["file"]))
        js, _, _ = O.run(inst, seed=0, passes=1, eps=0.0, theta=None)
        assert O.strip_time(js) == r["expected"][0], r["name"]
        if r["name"] in NAMES:
            (tmp_path / f"{r['name']}.json").write_text(js)
    for build in ("ref_cpu", "ref_host"):
        rc, text = compare_dirs(str(tmp_path), os.path.join(PARITY, build))
        assert rc == 0, text


def test_oracle_eps03_seeds_0_15_on_every_reference_instance():
    rows = [r for r in br_rows() if r["case"] == "eps03"]
    assert len(rows) == 20
    for r in rows:
        inst = O.OInstance(instance_text(r["file"]))
        for k, exp in zip(r["seeds"], r["restarts"]):
            js, _, _ = O.run(inst, seed=k, passes=1, eps=0.3, theta=0.9)
            assert row_digest(json.loads(js)) == exp[0], (r["name"], k)
            if k == 0:
                assert O.strip_time(js) == r["first"]
