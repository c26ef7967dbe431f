"""Regression fixture for the ring-removal kernels (run on a GPU).

Records remove_stripe_fw outputs of this library for the FW_CASES of
make_golden.py plus one odd-width db5 case.  The filter-bank stages add
tap by tap with round-to-nearest multiplies and adds in the reference's
order and the band FFTs are deterministic cuFFT plans, so any rewrite of the
filter-bank kernels that keeps that arithmetic reproduces these outputs bit
for bit (tests/test_gpu_stripe.py).  Usage:

    python tests/golden/make_fw_b200.py OUT.npz
"""
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))

from make_golden import FW_CASES, fw_input  # noqa: E402

CASES = FW_CASES + [(75, 3, 203, 5, 1.5, "db5", 6)]


def main(out):
    from tomocupy_b200.processing.remove_stripe import remove_stripe_fw
    res = {}
    for i, (nproj, nz, n, level, sigma, wname, seed) in enumerate(CASES):
        data = fw_input(nproj, nz, n, seed)
        res[f"in_{i}"] = data
        o = remove_stripe_fw(torch.as_tensor(data, device="cuda"), sigma, wname, level)
        res[f"out_{i}"] = o.cpu().numpy()
    np.savez_compressed(out, **res)
    print("wrote", out, len(CASES), "cases")


if __name__ == "__main__":
    main(sys.argv[1])
