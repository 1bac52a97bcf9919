import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    # always list the reasons of skipped tests in the summary (a test that
    # needs the reference checkout or a fixture says which)
    rc = getattr(config.option, "reportchars", None) or ""
    if "s" not in rc and "a" not in rc and "A" not in rc:
        config.option.reportchars = rc + "s"


def load_index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load_case(name, meta):
    """Returns (off, idx, wt, init, expected_labels_or_None, meta)."""
    from rbsc_b200 import graphs as G
    if meta["kind"] == "arrays":
        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        return (z["off"], z["idx"], z["wt"] if "wt" in z else None, z["init"] if "init" in z else None,
                z["labels"], meta)
    off, idx = getattr(G, meta["generator"])(**meta["kwargs"])
    return off, idx, None, None, None, meta


@pytest.fixture(scope="session")
def golden_index():
    return load_index()
