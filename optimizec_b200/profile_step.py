"""Short N-sized run used for ncu captures of the step kernels.

    python optimizec_b200/profile_step.py [N]

Initial field: k^4 exp(-2(k/K0)^2) spectrum, seed 1; NEXTDT; 1 + 3 steps.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import optimizec_b200 as P  # noqa: E402

N = int(sys.argv[1]) if len(sys.argv) > 1 else 4096
s = P.Solver(N, 1e5, 4.0, 0.1)
s.init_k4(1)
s.next_dt()
s.step(1)
s.next_dt()
s.step(3)
s.sync()
print("done", s.scalars()["it"])
