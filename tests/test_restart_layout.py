"""Restart files in the reference's own layout, checked on the CPU against
restart files the reference itself wrote (tests/golden/reference_restart_*:
RestartRegistrar::dumpState through FlatFileIO, src/DataOutput/
RestartRegistrar.cc:155-171, src/FileIO/FlatFileIO.cc)."""
import glob
import os

import numpy as np
import pytest

import flatfile

FIXTURES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "reference_restart_*.npz")))
IDS = [os.path.basename(p)[len("reference_restart_"):-4] for p in FIXTURES]


def test_fixtures_present():
    assert len(FIXTURES) >= 4


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_labels_match_the_reference(pkg, path):
    """The objects a dump writes, in order, under the registrar's unique
    labels (RestartRegistrar::uniqueLabels, :113-131), equal the reference's
    for the same configuration."""
    d = np.load(path)
    cfg = pkg.abi.SphConfig.from_buffer_copy(d["input/config"].tobytes())
    assert pkg.abi.restart_labels(cfg) == flatfile.labels(d["restart"].tobytes())


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_reference_file_layout(pkg, path):
    """What the reader relies on: every FieldList is a NodeListNames line
    ("name|" and a NUL, or empty) followed by its Field0 line, and a Field's
    count is the NodeList's node count."""
    d = np.load(path)
    e = flatfile.entries(d["restart"].tobytes())
    n = d["input/mass"].size
    for k, (p, raw) in enumerate(e):
        if p.endswith("/NodeListNames"):
            if raw == b"":
                continue
            assert raw == b"nodes|\0"
            nxt, vals = e[k + 1]
            assert nxt == p[:-len("NodeListNames")] + "Field0"
            assert int(flatfile.numbers(vals)[0]) == n
