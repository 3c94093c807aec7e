"""Load the golden fixtures written by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from uncc_sar_focusing_b200 import scenes as S

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The backprojection fixtures (pt_*.npz; the PGA fixtures pga_*.npz are
    read by the PGA tests)."""
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN_DIR, "pt_*.npz")))


def load(name):
    d = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    nx, ny, nz = (int(v) for v in d["grid"])
    x0, y0, z0, wx, wy, wz = (float(v) for v in d["grid_geom"])
    sc = S.Scene(name=name, phase_history=d["phase_history"], ant_x=d["ant_x"], ant_y=d["ant_y"],
                 ant_z=d["ant_z"], slant_range=d["slant_range"], start_freq=d["start_freq"],
                 delta_freq=float(d["delta_freq"]), nfft=int(d["nfft"]),
                 grid=S.Grid(nx=nx, ny=ny, nz=nz, x0=x0, y0=y0, z0=z0, wx=wx, wy=wy, wz=wz),
                 window=str(d["window"]))
    return sc, d
