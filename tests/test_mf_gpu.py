"""GPU matched filter (sarbp_matched_filter) against the FP64 oracle restatement
of matlab/mfBasic.m:73-89 (itself pinned to the reference's run_mf in
tests/test_oracle.py).  FP64 plans within 1e-9 (one ulp of a 10 km range,
2e-12 m, is 7e-10 rad of X-band phase, and the GPU contracts the sum of
squares into FMAs), mixed plans within 1e-4."""
import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import focusing

    return focusing


def scene(**kw):
    args = dict(K=64, Np=40, n=36, spacing=0.15, nfft=512, snr_db=20.0, seed=8, n_targets=4, extent=4.0)
    args.update(kw)
    return S.point_target_scene(**args)


def args(sc):
    return (sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_matched_filter_matches_oracle(F, precision, tol):
    sc = scene()
    want = O.mf_fp64(sc)
    with F.Plan.for_scene(sc, precision) as plan:
        got = plan.matched_filter(*args(sc))
    assert got.shape == want.shape
    assert O.rel_l2(got, want) < tol


def test_matched_filter_volume_no_taper_and_device_buffers(F):
    import torch

    sc = scene(K=48, Np=24, n=20, nfft=384)
    sc.window = None
    sc.grid = S.Grid(nx=20, ny=26, nz=3, wx=19 * 0.15, wy=25 * 0.15, wz=1.0, z0=0.2)
    want = O.mf_fp64(sc)
    with F.Plan.for_scene(sc, "mixed") as plan:
        host = plan.matched_filter(*args(sc))
        dev = plan.matched_filter(*(torch.as_tensor(np.ascontiguousarray(a)).cuda() for a in args(sc)))
        torch.cuda.synchronize()
    assert O.rel_l2(host, want) < 1e-4
    np.testing.assert_array_equal(dev.cpu().numpy(), host)


def test_matched_filter_and_backprojection_agree(F):
    """MF = nfft x BP up to backprojection's linear interpolation (8x
    oversampled range profiles: a few percent)."""
    sc = scene()
    with F.Plan.for_scene(sc, "mixed") as plan:
        mf = plan.matched_filter(*args(sc))
        bp = plan.focus(*args(sc))
    assert O.rel_l2(bp * sc.nfft, mf) < 0.03
