"""plp_block CLI: the drop-in for the reference's block-building engine
binaries (blockproof/plp_block.cpp, plp_block_cuda.cu). GPU tests compare its
output with the reference's own CPU build (oracle/_ref/plp_block), time_s
excluded as blockproof/run_cuda_parity.sh does."""
import json
import os
import subprocess
import tempfile

import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth

CLI = P.BLOCK_CLI_PATH
REF = os.path.join(O.REF_DIR, "plp_block")


def run(args):
    return subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)


@pytest.fixture(scope="module")
def files():
    d = tempfile.mkdtemp()
    out = []
    for k, inst in enumerate([synth.multi_restart(2), synth.batched(30001), synth.stress(40002)]):
        p = os.path.join(d, f"b{k}.txt")
        open(p, "w").write(inst.to_thpack())
        out.append(p)
    yield out


def test_usage_errors_exit_2(files):
    assert run([]).returncode == 2
    assert run([files[0], "--pick", "middle"]).returncode == 2
    assert run([files[0], "--bogus"]).returncode == 2
    assert run([files[0], "--device", "-3"]).returncode == 2


def test_instance_error_exits_1():
    r = run(["/nonexistent.txt", "--json"])
    assert r.returncode == 1 and r.stderr.startswith("instance error:")


def _strip(js):
    d = json.loads(js)
    d.pop("time_s")
    return d


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference block engine not built")
@pytest.mark.parametrize("cfg", [[], ["--amax", "4", "--bmax", "4", "--kmax", "6", "--eps", "0.5", "--topk", "64"],
                                 ["--pick", "contact"], ["--pick", "support", "--eps", "0", "--no-theta"]])
def test_json_and_fill_match_reference_cpu_build(files, cfg):
    for f in files:
        for seed in (0, 3):
            args = [f, "--seed", str(seed), "--single-pass", "--json"] + cfg
            a, b = run(args), subprocess.run([REF] + args, capture_output=True, text=True, timeout=300)
            assert a.returncode == 0 and b.returncode == 0, a.stderr
            assert _strip(a.stdout) == _strip(b.stdout)
            assert a.stderr.strip() == b.stderr.strip()          # fill_pct=...


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference block engine not built")
def test_text_mode_matches_reference_cpu_build(files):
    a = run([files[1], "--seed", "2", "--single-pass"])
    b = subprocess.run([REF, files[1], "--seed", "2", "--single-pass"], capture_output=True, text=True)
    strip = lambda s: s.split(" time_s=")[0]
    assert strip(a.stdout) == strip(b.stdout)


@pytest.mark.gpu
def test_device_rows_are_the_single_seed_runs(files):
    r = run([files[2], "--seed", "5", "--single-pass", "--device", "4", "--json"])
    assert r.returncode == 0, r.stderr
    rows = json.loads(r.stdout)["rows"]
    assert len(rows) == 4
    for k, row in enumerate(rows):
        one = run([files[2], "--seed", str(5 + k), "--single-pass", "--json"])
        row.pop("time_s")
        assert row == _strip(one.stdout)
