"""Direct-sum reference values for the precision-scaling study (CPU, float64).

Writes tests/golden/direct_sio2_{648,5184}.npz: energy [eV], forces [eV/A] and stress
[eV/A^3] of the direct pairwise D3(BJ) lattice sum (oracle/direct_d3.py, pairs within
25 A plus the continuum tail) for the seeded SiO2 box and its 2x2x2 replica with
N(0, 0.05 A) jitter (the same structures bench.py and the scaling study use).

    python tests/golden/make_direct.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fourierd3_b200 import structures as st  # noqa: E402
from oracle.direct_d3 import direct_calculate  # noqa: E402


def main():
    r_direct = 25.0
    for reps in (1, 2):
        if reps == 1:
            p, c, z = st.sio2_box(0)
        else:
            p, c, z = st.sio2_scaled(reps)
        e, f, s = direct_calculate(z, p, c, r_direct=r_direct, c6tol=1.0, r_cut=6.0)
        n = len(z)
        np.savez_compressed(os.path.join(HERE, f"direct_sio2_{n}.npz"), positions=p, cell=c, numbers=z,
                            energy_ev=np.float64(e), forces=f, stress=s, r_direct=np.float64(r_direct))
        print(n, e)


if __name__ == "__main__":
    main()
