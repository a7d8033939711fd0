"""The C restatement of the ply step (oracle/liboracle.so) against golden
digests recorded from the reference's own workers (tests/golden/)."""
import json
import os

import pytest

from oracle import oracle as orc
from tests.golden.scenarios import MATERIALS, run_material
from tests.parity import OracleSide

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ply_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.parametrize("material", MATERIALS)
def test_port_matches_reference_digests(golden, material):
    got = run_material(OracleSide(orc.Port(material)), material)
    bad = [k for k in got if json.loads(json.dumps(got[k])) != golden[k]]
    assert not bad, f"{len(bad)} scenarios differ, first: {bad[:3]}"
