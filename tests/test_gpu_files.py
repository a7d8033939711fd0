"""Per-ply files against the reference program's: tbgen -o writes the
reference's per-ply output (write_data's zstd frames, util.c:272-343, under
create_name's paths, kslice.c:306-315).  Every W and L directory of every
ply, the mates (0/L) and, after a whole generation, the final "wins"
(0/wins) -- read back as the reference's read_data reads them -- equal the
files the unmodified reference program writes for the same material and
7-piece stub (tests/golden/ply_files.json, made by
tests/golden/make_ply_files_golden.py), in resident and in streamed mode.
KRvK: the whole generation; KRvKN (five-valued stub: cursed wins and
blessed losses): the first 20 plies."""
import importlib.util
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TBGEN = os.path.join(ROOT, "tb8gen_b200", "tbgen")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ply_files.json")

_spec = importlib.util.spec_from_file_location(
    "ply_files_golden", os.path.join(ROOT, "tests", "golden", "make_ply_files_golden.py"))
_g = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_g)

CASES = [("KRvK", None), ("KRvKN", 20)]


@pytest.mark.parametrize("streamed", [False, True])
@pytest.mark.parametrize("material,max_ply", CASES)
def test_per_ply_files_equal_reference(tmp_path, material, max_ply, streamed):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    with open(GOLDEN) as f:
        golden = json.load(f)[material]
    out = tmp_path / "out"
    cmd = [TBGEN, "-q", "-o", str(out)]
    if golden["seed"] is not None:
        cmd += ["-s", str(golden["seed"]), "-m", str(golden["mod"])]
    if max_ply:
        cmd += ["-n", str(max_ply)]
    if streamed:
        cmd += ["-S"]
    r = subprocess.run(cmd + [material], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    mine = _g.digests(_g.zstd(), str(out))
    last = max(int(k.split("/")[0]) for k in mine)
    assert max_ply is None or last == max_ply
    compared = 0
    for key, ref in golden["dirs"].items():
        n = int(key.split("/")[0])
        if key.startswith("0/wins") and max_ply is not None:
            continue  # the final "wins" only after the whole generation
        if n > last:
            continue
        assert key in mine, f"{key} missing"
        assert mine[key] == ref, f"{key} differs"
        compared += 1
    extra = [k for k in mine if k not in golden["dirs"]]
    assert not extra, extra
    # the same directories as the reference (half-plies the schedule skips
    # have none), each with its 462 slices
    assert compared > 4 and all(mine[k][0] == 462 for k in mine)
