"""Generates tests/golden/complex_gamma.npz: complex arguments for the gamma
family, the reference's own complex outputs and mpmath values.

Run here, where the reference sources exist:

    REFERENCE_ROOT=<reference checkout> python oracle/build_ref.py
    python tests/golden/make_golden_complex.py

The reference's complex kernels are reached through its compiled CPU
operators (oracle/_ref/libtorchscience_ref.so: the reference's cpu/ kernels
instantiated over its headers), loaded alone in this process (this
package's library registers the same torch.ops namespace).  Truth is mpmath
1.3 at 30 digits: loggamma (the principal branch), gamma, psi(0), psi(1).
"""

from __future__ import annotations

import sys
from pathlib import Path

import mpmath as mp
import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
LIB = ROOT / "oracle" / "_ref" / "libtorchscience_ref.so"
OUT = Path(__file__).resolve().parent / "complex_gamma.npz"


def points():
    rng = np.random.default_rng(7)
    n = 1500
    z = [
        rng.uniform(-30, 30, n) + 1j * rng.uniform(-30, 30, n),  # bulk
        rng.uniform(0.1, 10, 300) + 1j * rng.uniform(-3, 3, 300),  # near the positive axis
        rng.uniform(-40, -0.1, 300) + 1j * rng.choice([-1, 1], 300) * 10.0 ** rng.uniform(-6, 0, 300),  # near the cut
        rng.uniform(-200, 200, 200) + 1j * rng.uniform(-200, 200, 200),  # large |z|
        rng.uniform(-5, 5, 200) + 1j * rng.choice([-1, 1], 200) * rng.uniform(15, 60, 200),  # large |Im z|
        np.array([1 + 0j, 2 + 0j, 0.5 + 0j, 1 + 1j, -0.5 + 0.5j, -8.5 + 1e-3j, -7.9 + 2j, -8.1 + 2j, 3 - 4j]),
    ]
    return np.concatenate(z)


def main():
    if not LIB.exists():
        raise SystemExit(f"{LIB} missing: build it with oracle/build_ref.py")
    torch.ops.load_library(str(LIB))
    z = points()
    zt = torch.from_numpy(z.astype(np.complex128))
    d = {"z": z}
    for name in ("log_gamma", "gamma", "digamma", "trigamma"):
        d[f"ref_{name}"] = getattr(torch.ops.torchscience, name)(zt).numpy()
    mp.mp.dps = 30
    conv = lambda f: np.array([complex(f(mp.mpc(complex(v)))) for v in z])  # noqa: E731
    d["truth_log_gamma"] = conv(mp.loggamma)
    d["truth_gamma"] = conv(mp.gamma)
    d["truth_digamma"] = conv(mp.digamma)
    d["truth_trigamma"] = conv(lambda v: mp.psi(1, v))
    d["truth_tetragamma"] = conv(lambda v: mp.psi(2, v))
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT.name}: {z.size} points")


if __name__ == "__main__":
    sys.exit(main())
