"""Generate tests/golden/: outputs of the reference's OWN kernels.

Runs the unmodified reference sgemm() (dispatching to sgemm_128x128x8 or
sgemm_128x256x8, src/sgemm.cuh:41-48) and sgemm_basic() (kernel_basic,
src/kernels/basic.cuh) -- built from the reference sources for sm_100a into
oracle/_ref/libref_sgemm.so by oracle/Makefile -- on inputs from the oracle's
seeded generator, and stores the outputs as raw float32 files plus index.json.
tests/test_oracle.py then pins the CPU oracle to these outputs.

Needs a B200.  Usage:  python tests/golden/make_golden.py [OUT_DIR]
(default: a new temporary directory, printed at the end; copy OUT_DIR/* into
tests/golden/ afterwards).
"""
import hashlib
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

# (name, m, n, k, alpha, beta, dist, which)  which: "sgemm" or "basic"
CASES = [
    ("t128_1x1x1", 1, 1, 1, 1.5, 0.5, 1, "sgemm"),
    ("t128_7x13x9", 7, 13, 9, 1.5, 0.5, 1, "sgemm"),
    ("t128_64x64x64_b0", 64, 64, 64, 1.0, 0.0, 0, "sgemm"),
    ("t128_128x128x8", 128, 128, 8, 1.5, 0.5, 0, "sgemm"),
    ("t128_129x257x33", 129, 257, 33, 1.5, 0.5, 0, "sgemm"),
    ("t128_300x200x100_pow2", 300, 200, 100, 1.5, 0.5, 2, "sgemm"),
    ("t128_200x136x1001", 200, 136, 1001, -0.75, 2.0, 0, "sgemm"),
    ("t256_2600x24x40", 2600, 24, 40, 1.5, 0.5, 0, "sgemm"),
    ("t256_2501x8x3", 2501, 8, 3, 1.5, 0.5, 1, "sgemm"),
    ("t256_40x2600x17_b0", 40, 2600, 17, 1.0, 0.0, 0, "sgemm"),
    ("basic_33x47x61", 33, 47, 61, 1.5, 0.5, 0, "basic"),
    ("basic_5x5x1", 5, 5, 1, 1.5, 0.5, 1, "basic"),
    ("basic_70x20x300_pow2", 70, 20, 300, 1.5, 0.5, 2, "basic"),
]
SEED = 20251203


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    dev = torch.device("cuda:0")
    index = []
    for name, m, n, k, alpha, beta, dist, which in CASES:
        A = oracle.fill(m, k, SEED, 1, dist)
        B = oracle.fill(k, n, SEED, 2, dist)
        C = oracle.fill(m, n, SEED, 3, dist)
        dA = torch.from_numpy(A).to(dev)
        dB = torch.from_numpy(B).to(dev)
        dC = torch.from_numpy(C).to(dev)
        oracle.ref_sgemm(dA, dB, dC, alpha, beta, basic=(which == "basic"))
        torch.cuda.synchronize()
        out = dC.cpu().numpy()
        fn = name + ".f32"
        out.tofile(os.path.join(out_dir, fn))
        if which == "basic":
            kernel = "kernel_basic"
        else:
            kernel = ("sgemm_128x256x8" if oracle.ref().ref_sgemm_kernel_choice(m, n)
                      else "sgemm_128x128x8")
        index.append({"name": name, "file": fn, "m": m, "n": n, "k": k, "alpha": alpha,
                      "beta": beta, "dist": dist, "seed": SEED, "ref_kernel": kernel,
                      "sha256": hashlib.sha256(out.tobytes()).hexdigest()})
        print(f"{name}: {kernel} done")
    with open(os.path.join(out_dir, "index.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "source": "reference sgemm()/sgemm_basic() built from its sources "
                             "for sm_100a (oracle/_ref), run on an NVIDIA B200",
                   "device": torch.cuda.get_device_name(0),
                   "cases": index}, f, indent=1)


if __name__ == "__main__":
    import tempfile

    out = sys.argv[1] if len(sys.argv) > 1 else tempfile.mkdtemp(prefix="sgemm_golden_")
    main(out)
    print(f"fixtures written to {out}")
