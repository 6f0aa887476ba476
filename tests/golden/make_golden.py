"""Generates tests/golden/lgl_kat.json: Legendre-Gauss-Lobatto nodes and weights for N=1..8
computed independently of the oracle and of the product (numpy's Legendre-series root finder
on P_N'(x), weights 2/(N(N+1) P_N(x)^2)).  Run: python tests/golden/make_golden.py
"""
import json
import os

import numpy as np
from numpy.polynomial import legendre as L


def lgl(N):
    c = np.zeros(N + 1)
    c[N] = 1.0
    inner = np.sort(np.real(L.legroots(L.legder(c)))) if N > 1 else np.array([])
    x = np.concatenate([[-1.0], inner, [1.0]])
    x = 0.5 * (x - x[::-1])  # exact symmetry
    PN = L.legval(x, c)
    w = 2.0 / (N * (N + 1) * PN ** 2)
    return x.tolist(), w.tolist()


if __name__ == "__main__":
    out = {str(N): dict(zip(("x", "w"), lgl(N))) for N in range(1, 9)}
    # closed forms for N=3 and N=4 (Abramowitz & Stegun 25.4.32) as an extra anchor
    out["closed_form"] = {
        "3": {"x": [-1.0, -1 / np.sqrt(5), 1 / np.sqrt(5), 1.0], "w": [1 / 6, 5 / 6, 5 / 6, 1 / 6]},
        "4": {"x": [-1.0, -np.sqrt(3 / 7), 0.0, np.sqrt(3 / 7), 1.0], "w": [0.1, 49 / 90, 32 / 45, 49 / 90, 0.1]},
    }
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lgl_kat.json")
    with open(p, "w") as f:
        json.dump(out, f, indent=1)
    print(p)
