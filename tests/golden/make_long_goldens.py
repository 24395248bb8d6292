"""Long-horizon fixtures computed by the CPU oracle (test infrastructure).

cfg1 of the benchmark configurations -- the plain method on a 51 x 51 stretched 2:1 channel,
first-order upwind, Re 100, beta 1, dt 1e-3, residual 1e-6, from rest plus seeded noise -- run by
the oracle for its full 200 physical steps.  The oracle restates the reference's loop in its
operation order (oracle/acs_oracle.cpp; pinned to the reference's own 51 x 84 run by
tests/test_oracle_golden.py).  The run takes several minutes on a few CPU cores, so its per-step
pseudo-iteration counts and final fields are stored once here and the GPU tests compare whole
200-step runs against them.

    python tests/golden/make_long_goldens.py [threads]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main(threads: int) -> None:
    import __graft_entry__ as entry
    from oracle import oracle as orc
    pkg = entry.load_package()
    pkg.configs.use_backend(orc)   # the oracle's own mesh and noise generators
    try:
        prm, mesh, st, itc, nsteps = pkg.configs.cfg_plain()
    finally:
        pkg.configs.use_backend(None)
    orc.set_threads(threads)
    case = orc.OracleCase(prm, mesh)
    s = {k: np.asfortranarray(v.copy()) for k, v in st.items()}
    t0 = time.time()
    itc, iters, err = case.run(s, nsteps, itc)
    keep = ("um", "vm", "p", "pn", "um_tau", "vm_tau")
    np.savez_compressed(os.path.join(HERE, "cfg1_plain51_200.npz"), iterations=np.asarray(iters, np.int64),
                        error=np.asarray(err), itc=itc, **{k: s[k] for k in keep})
    print(f"cfg1: {nsteps} steps, {int(np.sum(iters))} pseudo-iterations, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1))
