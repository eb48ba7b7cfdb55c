"""Generate the golden fixtures of the oracle tests from the REFERENCE
itself: the reference's kernel sources compiled in place (oracle/_ref, built
by oracle/Makefile from the IFOS2D source tree) are run on small seeded cases
and their outputs are stored here.  Run in a container that has the
reference tree:

    python tests/golden/make_golden.py [case ...]   (all cases and the set-up file when none are named)

The fixtures pin the C restatement (oracle/liboracle.so) bit-for-bit on
machines without the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tests.golden.cases import CASES, build_case  # noqa: E402


def main(names=None):
    O.build("ref")
    for name in names or CASES:
        p, model, g, sig, adj = build_case(name)
        out = O.run_shot("ref", p, model, g.srcpos, sig, g.recpos, run_adjoint=True, adj=adj)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), sections=out["sections"], fields=out["fields"],
                            grads=out["grads"], adj_fields=out["adj_fields"])
        print(name, {k: float(np.linalg.norm(v)) for k, v in out.items()})
    if names:
        return
    # set-up functions
    p, model, g, sig, adj = build_case("psv_el_o4")
    prof = {f"pml_fw{fw}": O.pml_profiles("ref", p.copy(fw=fw, npower=npw, vppml=v))
            for fw, npw, v in ((10, 2.0, 1800.0), (20, 4.0, 1700.0))}
    hc = np.stack([np.stack([O.fd_coeffs("ref", p.copy(fdorder=fd, maxrelerror=me)) for me in range(5)])
                   for fd in (2, 4, 6, 8, 10, 12)])
    wav = np.stack([O.wavelet("ref", p, shape, g.srcpos) for shape in (1, 2, 4, 5, 6, 8)])
    rng = np.random.default_rng(7)
    obs = rng.standard_normal((9, p.nt)).astype(np.float32)
    syn = rng.standard_normal((9, p.nt)).astype(np.float32)
    diff, l2, en, mf = O.calc_res("ref", p, obs, syn)
    np.savez_compressed(os.path.join(HERE, "setup.npz"), hc=hc, wavelets=wav, obs=obs, syn=syn, diff=diff,
                        sums=np.array([l2, en, mf]), **prof)


if __name__ == "__main__":
    main(sys.argv[1:])
