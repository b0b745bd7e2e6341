"""Regenerates tests/golden/oracle_golden.npz from the CPU oracle.

The reference ships no golden vectors for this path (its only FluidSim test is
unbuildable), so these fixtures pin the oracle itself against regressions:
a 12^3 sphere-pool system and its FP64 MIC(0)-PCG solution, and one P2G splat.
Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from helpers import poisson_system  # noqa: E402

O.build()
O.set_threads(1)
O.set_parity_mode(True)
n, seed = 12, 5
S = poisson_system(O, n, seed=seed)
p, res, it = O.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-8, max_iter=500,
                         criterion=O.CRIT_REL_L2)
rng = np.random.default_rng(9)
pos = rng.uniform(0.1, 0.9, (40, 3))
vel = rng.uniform(-1, 1, (40, 3))
out = O.p2g(pos, vel, (8, 8, 8), 1.0 / 8, flip=True)
np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), n=n, seed=seed, active=S["active"],
                    adiag=S["adiag"], pressure=p, iters=it, p2g_pos=pos, p2g_vel=vel,
                    p2g_u=out["u"], p2g_v=out["v"], p2g_w=out["w"], p2g_uw=out["uw"])
print("wrote", os.path.join(HERE, "oracle_golden.npz"), "iters", it)
