"""The committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py):
file integrity, and the FP64 oracle still reproducing every fixture from the same
seeded inputs (a regression pin on the oracle itself)."""
import hashlib
import json
import os
import sys

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_fixture_files_match_manifest():
    manifest = json.load(open(os.path.join(GOLDEN, "golden.json")))
    assert len(manifest) >= 10
    for name, digest in manifest.items():
        with open(os.path.join(GOLDEN, name), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == digest, name


def test_oracle_reproduces_the_fixtures(oracle):
    sys.path.insert(0, GOLDEN)
    import make_golden
    fresh = make_golden.cases()
    for name, arrays in fresh.items():
        stored = np.load(os.path.join(GOLDEN, name + ".npz"))
        assert set(stored.files) == set(arrays), name
        for k, v in arrays.items():
            np.testing.assert_allclose(stored[k], np.asarray(v), rtol=1e-12, atol=1e-14, err_msg=f"{name}:{k}")
