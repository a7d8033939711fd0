"""End-to-end known answers: whole generations by the C host driver
(tb8gen_b200/tbgen: calc_sub_kslices, calc_illegal_and_mate and the
calc_L_n / calc_W_n loop over the C ABI, all slices resident in HBM) print
the same per-ply counts as the unmodified reference program on the same
material (tests/golden/schedule_counts.json, made by
tests/golden/make_schedule_golden.py).  KRvK and KQvK are the reference's
real results (captures into KvK are draws); the others replace the 7-piece
probe by the seeded stub on both sides.  KRvKN uses the five-valued stub, so
cursed wins and blessed losses reach the ply-101 paths.  The resident
driver runs each half-ply as one recorded batch (the persistent kernel,
block-wide work items; -k 2: warp-wide); with -P it launches every call on
its own: all must print the golden counts."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "schedule_counts.json")
TBGEN = os.path.join(ROOT, "tb8gen_b200", "tbgen")

with open(GOLDEN) as f:
    CASES = json.load(f)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["batched", "batched-warp", "plain"])
@pytest.mark.parametrize("material", sorted(CASES))
def test_generation_counts_match_reference(material, path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    case = CASES[material]
    cmd = [TBGEN] + {"batched": [], "batched-warp": ["-k", "2"], "plain": ["-P"]}[path]
    if case["seed"] is not None:
        cmd += ["-s", str(case["seed"]), "-m", str(case["mod"])]
    r = subprocess.run(cmd + [material], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = [l.strip() for l in r.stdout.splitlines() if " = " in l]
    assert got == case["lines"]


STREAMED = [("KRvK", 16, False), ("KRRvK", 16, False), ("KRvKN", 16, False),
            ("KRRvKR", 16, False), ("KRvKN", 1, False), ("KRRvKR", 5, False),
            ("KQvKR", 64, False), ("KRvKN", 16, True), ("KRRvKR", 5, True), ("KQvKR", 32, True)]


@pytest.mark.parametrize("material,seg,host_wins", STREAMED)
def test_streamed_generation_counts_match_reference(material, seg, host_wins):
    """The same generations with the planes in host memory and a device
    window of slices that follows the schedule (tbgen -S), its steps run in
    pipelined segments of `seg` steps (reads, kernels and writes of adjacent
    segments overlap on three streams), the "wins" planes in HBM or, with
    -H, in the host tier too: identical counts."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    case = CASES[material]
    cmd = [TBGEN, "-S", "-g", str(seg)] + (["-H"] if host_wins else [])
    if case["seed"] is not None:
        cmd += ["-s", str(case["seed"]), "-m", str(case["mod"])]
    r = subprocess.run(cmd + [material], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    assert "streamed" in r.stderr
    got = [l.strip() for l in r.stdout.splitlines() if " = " in l]
    assert got == case["lines"]


@pytest.mark.parametrize("material", ["KRRvKR", "KQvKR"])
def test_streamed_slices_equal_resident(material):
    """Digests of 16 seeded slices of every half-ply's output (tbgen -c 16)
    are the same in resident mode, in the streamed pipeline and with the
    wins planes in the host tier: the modes agree slice by slice, not only
    in their counts."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    case = CASES[material]
    base = [TBGEN, "-c", "16"]
    if case["seed"] is not None:
        base += ["-s", str(case["seed"]), "-m", str(case["mod"])]
    outs = []
    for extra in ([], ["-S", "-g", "5"], ["-S", "-H"]):
        r = subprocess.run(base + extra + [material], capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr
        outs.append([l.strip() for l in r.stdout.splitlines() if " = " in l])
    sums = [l for l in outs[0] if l.startswith("sum ")]
    # one digest per half-ply: the count lines less the four of the set-up
    assert sums and len(sums) == len(outs[0]) - len(sums) - 4
    assert outs[1] == outs[0] and outs[2] == outs[0]
