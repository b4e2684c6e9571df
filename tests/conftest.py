import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, 'jax-power_b200')):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built library')
    config.addinivalue_line('markers', 'slow: CPU test that takes tens of seconds')
    config.addinivalue_line('markers', 'fullsize: GPU parity test on a benchmark configuration at its full '
                                       'size (512^3), with a CPU oracle run of a minute or two')
