import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    # temporary files of the tests (state files, built adapters) stay inside the checkout
    if not config.option.basetemp:
        os.makedirs(os.path.join(ROOT, "_build"), exist_ok=True)
        config.option.basetemp = os.path.join(ROOT, "_build", "pytest_tmp")
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size parity cases")
