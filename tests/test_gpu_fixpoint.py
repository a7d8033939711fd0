"""The fixpoint material against the reference program at every ply.

The unmodified reference program, with the seeded 7-piece stub (seed 1,
values mod 3), ran the whole generation of KQRvKRR (462 king slices, 101
plies) on the host cores; its per-ply count lines and the SHA-256 of every
W and L directory of its per-ply files are in
tests/golden/fixpoint_KQRvKRR.json (tests/golden/make_fixpoint_golden.py).
Here the C host driver runs the same generation on the GPU:

* streamed (planes in page-locked host memory, a device window of slices,
  the fixpoint bench's mode) and resident, each printing every count line of
  the reference's run;
* the first plies written as the reference's per-ply files (tbgen -o), every
  slice of every W and L directory equal to the reference's.
"""
import importlib.util
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TBGEN = os.path.join(ROOT, "tb8gen_b200", "tbgen")
GOLDEN = os.path.join(ROOT, "tests", "golden", "fixpoint_KQRvKRR.json")

_spec = importlib.util.spec_from_file_location(
    "ply_files_golden", os.path.join(ROOT, "tests", "golden", "make_ply_files_golden.py"))
_g = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_g)


@pytest.fixture(scope="module")
def golden():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(TBGEN):
        pytest.skip("tbgen not built")
    if not os.path.exists(GOLDEN):
        pytest.skip("tests/golden/fixpoint_KQRvKRR.json not recorded")
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.parametrize("streamed", [True, False])
def test_counts_every_ply_equal_reference(golden, streamed):
    cmd = [TBGEN, "-s", str(golden["seed"]), "-m", str(golden["mod"])]
    if streamed:
        cmd.append("-S")
    r = subprocess.run(cmd + [golden["material"]], capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    got = [l.strip() for l in r.stdout.splitlines() if " = " in l]
    assert len(got) == len(golden["counts"])
    bad = [(a, b) for a, b in zip(got, golden["counts"]) if a != b]
    assert not bad, bad[:5]


def test_first_plies_files_equal_reference(golden, tmp_path):
    max_ply = 8
    out = tmp_path / "out"
    cmd = [TBGEN, "-q", "-S", "-o", str(out), "-s", str(golden["seed"]), "-m",
           str(golden["mod"]), "-n", str(max_ply), golden["material"]]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    mine = _g.digests(_g.zstd(), str(out))
    compared = 0
    for key, ref in golden["dirs"].items():
        n = int(key.split("/")[0])
        if key.startswith("0/wins") or n > max_ply:
            continue
        assert key in mine, f"{key} missing"
        assert mine[key] == ref, f"{key} differs"
        compared += 1
    assert compared >= 4 * max_ply
