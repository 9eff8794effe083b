"""Write tests/golden/isf_16x8x8.npz: FP64 stage outputs of the ISF operators
on a seeded 16x8x8 jet-torus input, computed with oracle/matlabport.py (the
independent numpy restatement of src/MatlabPort.jl), not with the C++ oracle
they pin.

    python tests/golden/make_golden.py

The reference itself cannot run here (Julia is absent), and it holds no
golden vectors; these fixtures pin the oracle to a second, independent
formulation of the same operators.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import matlabport as mp  # noqa: E402
from helpers import smooth_psi  # noqa: E402

L = (4, 2, 2)
DIMS = (16, 8, 8)
HBAR = float(np.float32(0.1))
DT = float(np.float32(1 / 48))
CEN = tuple(float(np.float32(v)) for v in (2 - 1.7, 1 - 0.034, 1 + 0.066))
NLEN, NRAD = 0.5, 0.5
KVEC = (10.0, 0.0, 0.0)
OMEGA_T = float(np.float32(5.0 * DT))  # the oracle takes Float32 omgterm


def main():
    m = mp.MatlabISF(L, DIMS, HBAR, DT)
    psi = smooth_psi(DIMS, seed=1234)
    p1, p2 = mp.from_aos(psi)
    out = {"psi_in": psi}
    out["schroedinger_flow"] = mp.to_aos(*mp.schroedinger_flow(m, p1, p2))
    out["normalize"] = mp.to_aos(*mp.normalize(1.3 * p1, 1.3 * p2))
    v1 = mp.velocity_one_form(m, p1, p2, 1.0)
    out["one_form_hbar1"] = mp.vel_to_aos(*v1)
    out["one_form_hbar"] = mp.vel_to_aos(*mp.velocity_one_form(m, p1, p2, HBAR))
    f = mp.div(m, *v1)
    out["div"] = np.transpose(f, (2, 1, 0)).copy()
    out["poisson_q"] = np.transpose(mp.poisson_solve(m, f), (2, 1, 0)).copy()
    out["pressure_project"] = mp.to_aos(*mp.pressure_project(m, p1, p2))
    jet = mp.is_jet(m, CEN, NLEN, NRAD)
    out["isjet"] = np.transpose(jet, (2, 1, 0)).astype(np.uint8).copy()
    out["restrict_dot"] = mp.to_aos(*mp.restrict(m, p1, p2, jet, KVEC, OMEGA_T))
    rng = np.random.default_rng(99)
    parts = rng.uniform(0.05, 0.95, (256, 3)) * np.asarray(L, np.float64)
    parts[:8] = -1.0
    out["parts_in"] = parts
    q1, q2, pn = mp.jet_step(m, p1, p2, jet, KVEC, OMEGA_T, parts.copy())
    out["jet_step_psi"] = mp.to_aos(q1, q2)
    out["jet_step_parts"] = pn
    np.savez_compressed(os.path.join(HERE, "isf_16x8x8.npz"), **out)


if __name__ == "__main__":
    main()
