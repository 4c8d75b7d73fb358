"""Short runs used for ncu captures.

    python optimizec_b200/profile_step.py [N]      # step kernels: k^4 field (seed 1), NEXTDT, 1 + 3 steps
    python optimizec_b200/profile_step.py closure  # 3 closed steps at N=256 with a 6 x 32 network
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import numpy as np  # noqa: E402

import optimizec_b200 as P  # noqa: E402

arg = sys.argv[1] if len(sys.argv) > 1 else "4096"
if arg == "closure":
    s = P.Solver(256, 1e5, 4.0, 0.1)
    s.init_k4(1)
    s.next_dt()
    net = P.CNN(6, 32, seed=1)
    s.attach_closure(net, np.array([5.0, 1.0, 1.0, 0.01], np.float32), energy_check=1)
    s.step(3)
    s.sync()
    print("done", s.closure_stats())
else:
    N = int(arg)
    s = P.Solver(N, 1e5, 4.0, 0.1)
    s.init_k4(1)
    s.next_dt()
    s.step(1)
    s.next_dt()
    s.step(3)
    s.sync()
    print("done", s.scalars()["it"])
