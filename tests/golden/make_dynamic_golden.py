"""Golden vectors for the dynamic TDVP mode, from the reference's own Python
lineage (mqt-yaqs/src/mqt/yaqs/core/methods/tdvp.py:667-855,
local_dynamic_tdvp, the sweep its analog TJM uses, analog/analog_tjm.py:72).

Runs local_dynamic_tdvp of the vendored upstream, imported from the
reference tree with a stand-in for its `opt_einsum` dependency (not
installed here): `contract` becomes numpy.einsum with path optimisation,
which computes the same contractions.  Noise-free evolution from
|0...0>, dt = 0.05, 20 sweeps; after every sweep <Z_i> of the dense state
vector and the bond dimensions are written to dynamic_tdvp.csv.

Usage: python tests/golden/make_dynamic_golden.py /path/to/reference
"""
import csv
import os
import sys
import types

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("YAQS_REFERENCE_TREE")
if not REF:
    sys.exit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set YAQS_REFERENCE_TREE)")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from yaqs_julia_b200 import api  # noqa: E402

CASES = [
    # name, hamiltonian factory, L, chi_max, steps
    ("ising_disordered_chi4", lambda L: api.init_ising(L, [0.6, 1.2, 0.8, 1.4, 0.9, 1.1, 0.7],
                                                       [0.7, 1.3, 0.5, 1.1, 0.8, 1.2, 0.9, 0.6]), 8, 4, 20),
    ("heisenberg_h03_chi6", lambda L: api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3), 8, 6, 20),
    ("ising_g05_chi16", lambda L: api.init_ising(L, 1.0, 0.5), 8, 16, 20),
]
STATES = {"ising_disordered_chi4": "zeros", "heisenberg_h03_chi6": "Neel", "ising_g05_chi16": "wall"}


def _shim():
    oe = types.ModuleType("opt_einsum")

    def contract(*args, **kw):
        kw.pop("optimize", None)
        return np.einsum(*args, optimize=True)

    oe.contract = contract
    sys.modules["opt_einsum"] = oe


def main():
    _shim()
    sys.path.insert(0, os.path.join(REF, "mqt-yaqs", "src"))
    from mqt.yaqs.core.methods import tdvp

    rows = []
    for name, make_h, L, chi, steps in CASES:
        H = make_h(L)
        psi = api.MPS(L, state=STATES[name])
        # upstream layouts: MPS (d, left, right), MPO (d_out, d_in, left, right)
        state = types.SimpleNamespace(tensors=[t.transpose(1, 0, 2).copy() for t in psi.tensors], length=L,
                                      physical_dimensions=[2] * L)
        ham = types.SimpleNamespace(tensors=[w.transpose(1, 2, 0, 3).copy() for w in H.tensors], length=L)
        params = types.SimpleNamespace(dt=0.05, max_bond_dim=chi, threshold=1e-9, min_bond_dim=2)
        Zs = [None] * L

        def record(t):
            m = api.MPS(L, tensors=[x.transpose(1, 0, 2) for x in state.tensors])
            v = m.to_vec()
            v = v / np.linalg.norm(v)
            for i in range(L):
                if Zs[i] is None:
                    from oracle.dense import site_op
                    Zs[i] = site_op(api.Z, i + 1, L)
                rows.append([name, t, i + 1, float(np.real(np.vdot(v, Zs[i] @ v))),
                             ",".join(str(x.shape[2]) for x in state.tensors[:-1])])

        record(0)
        for t in range(1, steps + 1):
            tdvp.local_dynamic_tdvp(state, ham, params)
            record(t)
    with open(os.path.join(HERE, "dynamic_tdvp.csv"), "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["Case", "Step", "Site", "Z", "Bonds"])
        w.writerows(rows)


if __name__ == "__main__":
    main()
