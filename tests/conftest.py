import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine")


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def golden_input(case):
    """Input rows of a golden case, rebuilt from its recorded source."""
    import parallel_ra_b200 as P
    src = case["source"]
    if src[0] == "fixture":
        rows = P.datagen.read_relation(os.path.join(GOLDEN, f"{src[1]}_edge_2_1_2"))
    elif src[0] == "er":
        rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(src[1], src[2], src[3]))
    elif src[0] == "tree":
        rows = P.datagen.with_row_ids(P.datagen.random_tree(src[1], src[2]))
    else:
        raise ValueError(src)
    return rows


def rows_digest(rows):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u8").tobytes()).hexdigest()


# graph-program cases (make_golden.py's manifest); the generated analyses of
# make_slog_golden.py have their own tests (test_wide.py)
with open(os.path.join(GOLDEN, "manifest.json")) as _f:
    _ALL = sorted(json.load(_f))
# the benchmark inputs (tc-er22, sg-tree15): minutes of CPU time on the reference and
# the oracle, so they have their own GPU tests (test_scale_parity.py)
LARGE_CASES = ("er4194304_tc", "tree32768_sg")
GOLDEN_CASES = [c for c in _ALL if c not in LARGE_CASES]
LARGE_GOLDEN = [c for c in _ALL if c in LARGE_CASES]
