"""Write tests/golden/born_u5_m6.json: counts, matrix checksums and energies of
the CPU oracle on the Born sphere (box +-8 A, uniform level 5, surface level 6).

The reference cannot be built here and ships no golden outputs; this fixture
pins the oracle against its own earlier output so regressions show up, while
its physics is pinned by the analytic Born energy (tests/test_oracle_cpu.py).
Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from cudanextgenpb_b200 import build, configs  # noqa: E402
from oracle_lib import Oracle  # noqa: E402


def main():
    build.build_all()
    prob = configs.make_born_problem(5, 6).build()
    info = prob.info()
    o = Oracle(prob)
    marker, border = o.markers()
    o.density()
    rp, col, val, rhs = o.assemble()
    phi, it, rel = o.solve("cg", 1e-12)
    e = o.energy()
    out = {
        "config": "Born sphere q=+1 a=2 A, box [-8,8]^3, unilevel 5, maxlevel 6, bc_type 3",
        "mesh_counts": [info["n_oct"], info["n_nodes"], info["n_hang"]],
        "n_border": int(len(border)),
        "nnz": int(rp[-1]),
        "sum_val": float(val.sum()),
        "sum_rhs": float(rhs.sum()),
        "energy": {k: e[k] for k in ("energy_pol", "energy_react", "charge_flux", "sum")},
        "analytic_born_kT": configs.born_energy(),
    }
    with open(os.path.join(HERE, "born_u5_m6.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
