"""Generate gaus_golden.npz: values of the reference's own Python restatement
of GAUS (tests/init/visualize_gaussian.ipynb, function calculate_gaussian, the
perturbed Gaussian of mod_layout.f90:640-672) at fixed points, for parameter
sets that use the z-waviness (DX, DY, K, DP) and the core modulation (DR, RK,
RP).  The oracle's GAUS is checked against these values on the CPU.

Run from the repository root where the reference tree is available:
    python tests/golden/make_gaus_golden.py /path/to/MLegS
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PARAMS = [
    dict(Q=1.0, B=1.0, R=1.0, XC=0.0, YC=0.0, K=1.0, RK=0.0, DX=0.0, DY=0.0, DR=0.0, DP=0.0, RP=0.0,
         ZLEN=2 * np.pi),
    dict(Q=0.5, B=1.5, R=0.8, XC=0.4, YC=-0.3, K=2.0, RK=1.0, DX=0.05, DY=-0.02, DR=0.1, DP=30.0, RP=-45.0,
         ZLEN=5.0),
    dict(Q=-2.0, B=0.7, R=1.3, XC=-1.0, YC=0.6, K=3.0, RK=2.0, DX=0.2, DY=0.1, DR=0.3, DP=90.0, RP=10.0,
         ZLEN=2 * np.pi),
]


def load_reference_function(root):
    nb = json.load(open(os.path.join(root, "tests", "init", "visualize_gaussian.ipynb")))
    for cell in nb["cells"]:
        src = "".join(cell.get("source", []))
        if "def calculate_gaussian" in src:
            lines = src.splitlines()
            start = next(i for i, l in enumerate(lines) if l.startswith("def calculate_gaussian"))
            body = [lines[start]]
            for l in lines[start + 1:]:
                if l and not l.startswith((" ", "\t")):
                    break
                body.append(l)
            ns = {"np": np}
            exec("\n".join(body), ns)
            return ns["calculate_gaussian"]
    raise RuntimeError("calculate_gaussian not found")


def main(root):
    f = load_reference_function(root)
    rng = np.random.default_rng(2024)
    x = rng.uniform(-3.0, 3.0, 64)
    y = rng.uniform(-3.0, 3.0, 64)
    z = rng.uniform(0.0, 5.0, 64)
    keys = ["Q", "B", "R", "XC", "YC", "K", "RK", "DX", "DY", "DR", "DP", "RP", "ZLEN"]
    params = np.array([[p[k] for k in keys] for p in PARAMS])
    vals = np.array([[f(x[i], y[i], z[i], p) for i in range(x.size)] for p in PARAMS])
    np.savez(os.path.join(HERE, "gaus_golden.npz"), keys=np.array(keys), params=params, x=x, y=y, z=z, vals=vals)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MLEGS_REFERENCE", "."))
