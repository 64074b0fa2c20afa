"""The oracle against its committed regression fixtures
(tests/golden/oracle_regression.json, written by
tests/golden/make_oracle_regression.py): every bit of every state field after
four steps of nine seeded decks, across the widened physics.  The reference
itself cannot be run here (no Fortran compiler), so these pin the
restatement against unintended change; the GPU path is held to the oracle
bit for bit by the GPU parity tests."""
import importlib.util
import json
import os

import pytest

from conftest import ROOT

HERE = os.path.join(ROOT, "tests", "golden")


def _maker():
    spec = importlib.util.spec_from_file_location("make_oracle_regression",
                                                  os.path.join(HERE, "make_oracle_regression.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


GOLD = json.load(open(os.path.join(HERE, "oracle_regression.json")))


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
def test_oracle_matches_its_fixture(name):
    mk = _maker()
    got = mk.run(mk.cases()[name])
    want = GOLD["cases"][name]
    for f in mk.STATE:
        assert got[f]["sha256"] == want[f]["sha256"], f"{name}: {f} changed (sum {got[f]['sum']} vs {want[f]['sum']})"
    assert got["_scalars"] == want["_scalars"]
