"""The two golden records of the reference program's runs agree: every
count line "w<n>_<c>" / "l<n>_<c>" of tests/golden/schedule_counts.json has
its directory <n>/W|L/<c> among the per-ply file digests of
tests/golden/ply_files.json and the other way round, and every directory
holds the 462 king slices.  CPU only."""
import json
import os
import re

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_ply_file_digests_match_count_lines():
    counts = json.load(open(os.path.join(HERE, "schedule_counts.json")))
    files = json.load(open(os.path.join(HERE, "ply_files.json")))
    for mat, rec in files.items():
        assert counts[mat]["seed"] == rec["seed"] and counts[mat]["mod"] == rec["mod"]
        want = set()
        for line in counts[mat]["lines"]:
            m = re.match(r"([wl])(\d+)_([wb]) = ", line)
            if m and int(m.group(2)) > 0:
                want.add(f"{m.group(2)}/{m.group(1).upper()}/{m.group(3)}")
        got = {k for k in rec["dirs"] if not k.startswith("0/")}
        assert got == want, mat
        assert {"0/L/w", "0/L/b", "0/wins/w", "0/wins/b"} <= set(rec["dirs"])
        assert all(n == 462 for n, _ in rec["dirs"].values())
