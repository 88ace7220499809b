import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "verb-4d_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests", "golden"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as O

    O.build(with_ref=None)
    return O.oracle()


@pytest.fixture(scope="session")
def gpu():
    import torch  # noqa: F401  (device presence check only)

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from verb4d_b200 import _lib

    return _lib.load()
