import os
import sys

# The oracle's numpy uses OpenBLAS built with MAX_THREADS=64; on hosts with more cores
# its multithreaded complex GEMM (n >= 128) has returned wrong results.  Cap the threads
# before numpy loads, and again at run time in case a plugin imported it first.
for _v in ('OPENBLAS_NUM_THREADS', 'OMP_NUM_THREADS', 'MKL_NUM_THREADS'):
    os.environ.setdefault(_v, '8')

import pytest  # noqa: E402

try:
    from threadpoolctl import threadpool_limits

    threadpool_limits(8)
except ImportError:  # pragma: no cover
    pass

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')
    config.addinivalue_line('markers', 'slow: longer CPU oracle runs')


@pytest.fixture(scope='session')
def cuda_device():
    import torch

    assert torch.cuda.is_available(), 'GPU test run without a CUDA device'
    return torch.device('cuda', 0)
