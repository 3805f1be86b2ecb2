import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "oracle", "large-strain-matrix-free_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture
def parity(request):
    """record(name, observed, bound): note an observed parity error beside its
    bound.  With LSMF_PARITY_LOG=<file> set, each record is appended to that
    file as one JSON line (test id, name, observed, bound), so a GPU run of
    the suite produces the table of observed errors."""
    import json
    path = os.environ.get("LSMF_PARITY_LOG")

    def record(name, observed, bound):
        if path:
            with open(path, "a") as f:
                f.write(json.dumps({"test": request.node.nodeid, "name": name, "observed": float(observed),
                                    "bound": float(bound)}) + "\n")
    return record
