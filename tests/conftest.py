import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def rel_l2(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is available")
    return torch.device("cuda")


@pytest.fixture(scope="session")
def ref():
    """The reference CUDA build (oracle/_ref) driven through oracle.refglue."""
    from oracle import refglue
    if not refglue.available():
        pytest.fail("oracle/_ref is not built: run `make -C oracle` (needs the reference sources)")
    return refglue


class TorchCuFFT:
    """Real FFTs through cuFFT (torch.fft on the GPU), the library that the
    reference's cupy.fft calls, with NumPy's types (float32 <-> complex64,
    float64 <-> complex128) and normalisation; a drop-in ``fft`` provider for
    the oracle's ring-removal restatements."""

    @staticmethod
    def rfft(a, axis=-1):
        import numpy as np
        import torch
        x = torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        return torch.fft.rfft(x, dim=axis).cpu().numpy()

    @staticmethod
    def irfft(a, n, axis=-1):
        import numpy as np
        import torch
        x = torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        return torch.fft.irfft(x, n=n, dim=axis).cpu().numpy()
