"""Regenerates tr_het_32x32.npz: the oracle's time-reversal image for the
heterogeneous, absorbing 32^2 case of tests/test_gpu_time_reversal.py
(oracle/tr.py, DOP853 at rtol = atol = 1e-12).  Run from the repository root:
    python tests/golden/make_tr_het.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main():
    import test_gpu_time_reversal as t
    from oracle import ode as oo
    from oracle import tr as otr

    dom, ts, ddom, dwpt, src, img, data, cgrid = t.het_setup()
    odom, owpt, osrc = t._oracle_objects(ddom, dwpt, src, dom)
    speed = oo.GridSpeed(cgrid, dom.dx, method="bspline3", boundary="clamp")
    image, _ = otr.time_reversal(data, odom, owpt, osrc, speed, np.asarray(img.positions), dom.grid_size, 200,
                                 lam=t.LAM_HET)
    np.savez_compressed(os.path.join(HERE, "tr_het_32x32.npz"), data=data, image=image)


if __name__ == "__main__":
    main()
