"""plp_gpu CLI: the drop-in for the reference plp_gpu / plp_gpu_cuda binaries.

CPU tests cover the paths that end before any CUDA call (usage errors exit 2,
instance errors exit 1, --selftest); GPU tests compare the JSON of every mode
with the reference's own g++ build (oracle/_ref/plp_gpu) and the reference
decoder running on this library's feasibility kernel (oracle/_ref/plp_gpu_capi),
time_s excluded as parity/compare_parity.py:30-31 does.
"""
import json
import os
import subprocess
import tempfile

import pytest

import oracle_py as O
import plpb200 as P
from conftest import GOLDEN
from plpb200 import synth

CLI = P.CLI_PATH
REF_HOST = os.path.join(O.REF_DIR, "plp_gpu")
REF_CAPI = os.path.join(O.REF_DIR, "plp_gpu_capi")


def run(args, **kw):
    return subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300, **kw)


@pytest.fixture(scope="module")
def inst_file():
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(synth.single_pass(1).to_thpack())
    yield f.name
    os.unlink(f.name)


# ------------------------------------------------------------------ CPU paths
def test_selftest_matches_cpython():
    r = run(["--selftest"])
    assert r.returncode == 0
    assert r.stdout == open(os.path.join(GOLDEN, "selftest_ref.txt")).read()


@pytest.mark.parametrize("args", [[], ["--bogus"], ["a.txt", "b.txt"], ["x.txt", "--seed"]])
def test_usage_errors_exit_2(args):
    assert run(args).returncode == 2


def test_bad_order_and_batch_flags_exit_2(inst_file):
    assert run([inst_file, "--order", "random"]).returncode == 2
    assert run([inst_file, "--batch", "4"]).returncode == 2            # needs --json
    assert run([inst_file, "--batch", "4", "--device", "4", "--json"]).returncode == 2


def test_instance_errors_exit_1():
    r = run(["/nonexistent/instance.txt", "--json"])
    assert r.returncode == 1 and r.stderr.startswith("instance error:")
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write("1\n1 1\n587 0 220\n1\n1 10 1 20 1 30 1 5\n")
    r = run([f.name, "--json"])
    os.unlink(f.name)
    assert r.returncode == 1
    assert r.stderr.strip() == "instance error: container dimensions must be positive"


# ------------------------------------------------------------------ GPU parity
def _strip(js):
    d = json.loads(js)
    d.pop("time_s")
    return d


def _ref(args):
    out = subprocess.run([REF_HOST] + args, capture_output=True, text=True, check=True, timeout=300)
    return _strip(out.stdout)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [["--single-pass", "--eps", "0", "--no-theta"],
                                   ["--single-pass", "--seed", "3"],
                                   ["--single-pass", "--seed", "2", "--order", "input"],
                                   ["--single-pass", "--first-fit", "--theta", "0.5"]])
def test_cli_single_run_matches_reference_host(inst_file, flags):
    if not os.path.exists(REF_HOST):
        pytest.skip("reference host build not present")
    for mode in ([], ["--plain"]):
        r = run([inst_file, "--json"] + flags + mode)
        assert r.returncode == 0, r.stderr
        assert _strip(r.stdout) == _ref([inst_file, "--json"] + flags)


@pytest.mark.gpu
def test_cli_device_and_batch_rows_match_reference_per_seed(inst_file):
    if not os.path.exists(REF_HOST):
        pytest.skip("reference host build not present")
    for mode in ("--device", "--batch"):
        r = run([inst_file, "--json", "--single-pass", mode, "24", "--seed", "5"])
        assert r.returncode == 0, r.stderr
        d = json.loads(r.stdout)
        assert d["K"] == 24 and d["n_passes"] == 1 and len(d["rows"]) == 24
        for k in (0, 7, 23):
            row = dict(d["rows"][k])
            row.pop("time_s")
            assert row == _ref([inst_file, "--json", "--single-pass", "--seed", str(5 + k)])


@pytest.mark.gpu
def test_cli_rngdump_passes():
    r = run(["--rngdump", "64"])
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip().endswith("RNGDUMP: PASS")


@pytest.mark.gpu
def test_reference_decoder_on_capi_backend_matches_reference_host():
    """The binding a reference maintainer would add (oracle/ref_backend_capi.cpp)."""
    if not (os.path.exists(REF_HOST) and os.path.exists(REF_CAPI)):
        pytest.skip("reference builds not present")
    for inst in (synth.single_pass(1), synth.multi_restart(2), synth.stress(40005)):
        with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
            f.write(inst.to_thpack())
        for flags in (["--eps", "0", "--no-theta"], ["--seed", "9"]):
            out = subprocess.run([REF_CAPI, f.name, "--single-pass", "--json"] + flags, capture_output=True,
                                 text=True, check=True, timeout=600)
            assert _strip(out.stdout) == _ref([f.name, "--single-pass", "--json"] + flags)
        os.unlink(f.name)


@pytest.mark.gpu
def test_time_budget_on_device_equals_fixed_passes(inst_file):
    """--time S without --single-pass runs passes on the device until S has
    elapsed (the reference's run loop); the packing equals a fixed run of the
    pass count it reports."""
    r = run([inst_file, "--time", "0.01", "--seed", "3", "--json"])
    assert r.returncode == 0, r.stderr
    d = _strip(r.stdout)
    n = d["n_passes"]
    assert n >= 2
    fixed = run([inst_file, "--passes", str(n), "--seed", "3", "--json"])
    assert fixed.returncode == 0
    assert _strip(fixed.stdout) == d


def _multi_text(insts):
    """One thpack file holding several instances (P = len(insts))."""
    body = ["".join(i.to_thpack().splitlines(keepends=True)[1:]) for i in insts]
    return f"{len(insts)}\n" + "".join(body)


def test_multi_instance_file_needs_the_flag():
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(_multi_text([synth.single_pass(1), synth.batched(30001)]))
    r = run([f.name, "--json"])
    os.unlink(f.name)
    assert r.returncode == 1
    assert r.stderr.strip() == "instance error: expected exactly 1 instance, got 2"


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [["--single-pass"], ["--device", "4", "--single-pass"]])
def test_multi_instance_file_in_one_launch(extra):
    insts = [synth.single_pass(1), synth.batched(30001), synth.batched(30002)]
    with tempfile.TemporaryDirectory() as d:
        multi = os.path.join(d, "multi.txt")
        open(multi, "w").write(_multi_text(insts))
        r = run([multi, "--multi", "--json", "--seed", "2"] + extra)
        assert r.returncode == 0, r.stderr
        lines = r.stdout.strip().splitlines()
        assert len(lines) == len(insts)
        for i, inst in enumerate(insts):
            one = os.path.join(d, f"one{i}.txt")
            open(one, "w").write(inst.to_thpack())
            single = run([one, "--json", "--seed", "2"] + extra)
            assert single.returncode == 0
            a, b = json.loads(lines[i]), json.loads(single.stdout)
            if "rows" in a:
                a, b = [_strip(json.dumps(x)) for x in a["rows"]], [_strip(json.dumps(x)) for x in b["rows"]]
            else:
                a, b = _strip(lines[i]), _strip(single.stdout)
            assert a == b
            if "--device" not in extra:
                assert a == _ref([one, "--json", "--seed", "2", "--single-pass"])


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "plp_gpu_cuda")),
                    reason="reference CUDA build not present")
@pytest.mark.parametrize("flags", [["--single-pass"], ["--single-pass", "--eps", "0", "--no-theta"]])
def test_reference_cuda_build_rows_equal_ours(inst_file, flags):
    """The reference's own CUDA build (--device K, its persistent kernel) on
    the same GPU gives the rows this library gives."""
    ref = subprocess.run([os.path.join(O.REF_DIR, "plp_gpu_cuda"), inst_file, "--device", "8", "--json",
                          "--seed", "4"] + flags, capture_output=True, text=True, check=True, timeout=300)
    ours = run([inst_file, "--device", "8", "--json", "--seed", "4"] + flags)
    assert ours.returncode == 0
    a, b = json.loads(ref.stdout)["rows"], json.loads(ours.stdout)["rows"]
    for x, y in zip(a, b):
        x.pop("time_s")
        y.pop("time_s")
    assert a == b and len(a) == 8
